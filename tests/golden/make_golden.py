"""Generate the committed golden fixtures from the REFERENCE itself.

Run in a container that holds the reference sources (default
/root/reference) after ``sh oracle/build_ref.sh``:

    python tests/golden/make_golden.py [reference_dir]

Outputs (numpy .npz, float64):
  wall.npz   -- the reference's own fixture tests-wall.pos (300 charges,
                L = 10) with the total-force columns 2-4 of tests-wall.for,
                plus the reference's P3M forces for every method on it and
                its influence functions / ad self-force coefficients.
  sweep.npz  -- a seeded 1000-particle uniform system in a box of side 10
                (system_type 0, charges +-1 alternating) with the reference's
                method-7 forces (mesh 16, cao 7, rcut 3, mc 2) at three alphas
                of the 0.1..2.5 step 0.05 sweep, and its Ewald forces.
  cli/*.dat  -- the out.dat tables of the reference program (oracle/_ref/p3m)
                for the command lines in CLI_CASES, each with its own
                generated system and Ewald reference forces.
The GPU box never runs this script; tests read the .npz files only.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "p3m-standalone_b200"))

import oracle as O  # noqa: E402
import p3mg  # noqa: E402

# (method, mesh, cao, mc, alpha, rcut) per method on the wall system
WALL_CASES = [
    (0, 16, 7, 2, 1.1, 3.0),
    (1, 16, 5, 1, 1.0, 3.0),
    (2, 16, 7, 2, 1.2, 3.0),
    (3, 12, 4, 1, 0.9, 3.0),
    (6, 16, 6, 1, 1.1, 3.0),
    (7, 16, 7, 2, 1.1, 3.0),
]


# command lines of the reference program whose out.dat tables are kept
CLI_CASES = {
    "m7_type0": "particles 300 box 8 mesh 12 cao 5 rcut 2.5 method 7 mc 2 alphamin 0.5 alphamax 1.5 "
                "alphastep 0.25 error_k",
    "m1_type3": "particles 300 box 8 mesh 12 cao 5 rcut 2.5 method 1 system_type 3 alphamin 0.5 alphamax 1.5 "
                "alphastep 0.25 error_k",
    "m0_type5": "particles 400 box 9 mesh 16 cao 3 rcut 2.5 method 0 system_type 5 alphamin 0.6 alphamax 1.4 "
                "alphastep 0.2 error_k",
    "m3_type1": "particles 300 box 8 mesh 14 cao 4 rcut 2.5 method 3 system_type 1 alphamin 0.8 alphamax 1.2 "
                "alphastep 0.2 mc_est 2",
    "m6_type4": "particles 300 box 8 mesh 12 cao 6 rcut 2.5 method 6 system_type 4 alphamin 0.8 "
                "alphamax 1.2 alphastep 0.2",
    "m2_type2": "particles 216 box 8 mesh 12 cao 7 rcut 2.5 method 2 system_type 2 alphamin 0.9 alphamax 1.3 "
                "alphastep 0.2",
}


def make_cli_goldens():
    import subprocess
    import tempfile
    exe = os.path.join(ROOT, "oracle", "_ref", "p3m")
    os.makedirs(os.path.join(HERE, "cli"), exist_ok=True)
    for name, args in CLI_CASES.items():
        with tempfile.TemporaryDirectory() as tmp:
            out = os.path.join(tmp, "out.dat")
            subprocess.run([exe] + args.split() + ["outfile", out], cwd=tmp, check=True, stdout=subprocess.DEVNULL,
                           stderr=subprocess.DEVNULL)
            with open(out) as f:
                text = f.read()
        with open(os.path.join(HERE, "cli", name + ".dat"), "w") as f:
            f.write("# " + args + "\n" + text)


def main(ref_dir):
    if not O.ref_available():
        raise SystemExit("oracle/_ref/libp3mref.so missing: run sh oracle/build_ref.sh first")
    x, y, z, q, L = p3mg.read_system(os.path.join(ref_dir, "tests-wall.pos"))
    n = len(x)
    ewald_for = p3mg.read_exact_forces(os.path.join(ref_dir, "tests-wall.for"), n)
    out = dict(x=x, y=y, z=z, q=q, L=L, for_total=ewald_for, cases=np.array(WALL_CASES, dtype=np.float64))
    for k, (m, mesh, cao, mc, alpha, rcut) in enumerate(WALL_CASES):
        r = O.ref_forces(m, mesh, cao, mc, alpha, rcut, x, y, z, q, L, want_G=True)
        out["f_%d" % k] = r["f"]
        out["fk_%d" % k] = r["f_k"]
        out["fr_%d" % k] = r["f_r"]
        out["energy_%d" % k] = r["energy"]
        out["G_%d" % k] = r["G"]
        if m in (2, 7):
            out["self_%d" % k] = O.ref_self_force_coeffs(m, mesh, cao, mc, alpha, x, y, z, q, L)
    np.savez_compressed(os.path.join(HERE, "wall.npz"), **out)

    # config-1-like sweep system
    x, y, z, q = p3mg.generate_system(0, 1000, 10.0, seed=12345)
    alphas = p3mg.alpha_sweep(0.1, 2.5, 0.05)
    pick = [alphas[0], alphas[24], alphas[-1]]
    out = dict(x=x, y=y, z=z, q=q, L=10.0, alphas=np.array(pick), n_alphas=len(alphas))
    for k, a in enumerate(pick):
        r = O.ref_forces(7, 16, 7, 2, a, 3.0, x, y, z, q, 10.0)
        out["f_%d" % k] = r["f"]
        out["fk_%d" % k] = r["f_k"]
    e = O.ref_ewald(x, y, z, q, 10.0, 16)
    out["ewald_f"] = e["f"]
    out["ewald_alpha"] = e["alpha"]
    out["ewald_kmax"] = e["kmax"]
    np.savez_compressed(os.path.join(HERE, "sweep.npz"), **out)
    make_cli_goldens()
    print("wrote", os.path.join(HERE, "wall.npz"), os.path.join(HERE, "sweep.npz"), os.path.join(HERE, "cli"))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
