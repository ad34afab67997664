"""Generate the committed golden fixtures from the REFERENCE itself.

Run in a container that holds the reference sources, after
``sh oracle/build_ref.sh <reference_dir>``:

    python tests/golden/make_golden.py <reference_dir>
    (or set P3M_REFERENCE_DIR and omit the argument)

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
                generated system and Ewald reference forces; cli/*.inhomo,
                *.map, *.map2d the inhomo_output and error map files the
                program writes beside them.
  inhomo.npz -- the reference's inhomogeneous error estimate and error map
                (INHOMO_CASES, ERROR_MAP_CASES) on a seeded 200-particle
                system.
  vincent.npz -- raw text of the reference's data sets
                (Data/ReferenceDataVincent, VINCENT_FILES): NaCl snapshots
                and a water box with their exact Ewald forces.
Single parts: --cli <case>..., --inhomo or --vincent [reference_dir].
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
    # inhomogeneous estimate (err_inhomo column, inhomo_output file)
    "m2_inhomo": "particles 200 box 6 mesh 12 cao 5 rcut 2.5 method 2 alphamin 0.9 alphamax 1.1 alphastep 0.2 "
                 "error_k inhomo_error inhomo_mesh 8 inhomo_cao 5 inhomo_mc 1 inhomo_output inhomo.txt",
    # error map files.  A single alpha: the reference opens error_map.dat and
    # error_map_2d.dat once per alpha and never closes them (main.c:407-423),
    # so with several alphas the earlier streams' buffers are flushed over
    # the last alpha's contents at exit.
    "m2_errmap": "particles 200 box 6 mesh 12 cao 5 rcut 2.5 method 2 alphamin 1.1 alphamax 1.1 alphastep 0.2 "
                 "error_k error_map error_map_mesh 8 error_map_cao 3",
}

# files the program writes next to out.dat, kept as <case>.<suffix>
CLI_EXTRA_FILES = {"inhomo.txt": "inhomo", "error_map.dat": "map", "error_map_2d.dat": "map2d"}


def make_cli_goldens(names=None):
    import subprocess
    import tempfile
    exe = os.path.join(ROOT, "oracle", "_ref", "p3m")
    os.makedirs(os.path.join(HERE, "cli"), exist_ok=True)
    for name, args in CLI_CASES.items():
        if names and name not in names:
            continue
        extra = {}
        with tempfile.TemporaryDirectory() as tmp:
            out = os.path.join(tmp, "out.dat")
            subprocess.run([exe] + args.split() + ["outfile", out], cwd=tmp, check=True, stdout=subprocess.DEVNULL,
                           stderr=subprocess.DEVNULL)
            with open(out) as f:
                text = f.read()
            for fname, suffix in CLI_EXTRA_FILES.items():
                if os.path.exists(os.path.join(tmp, fname)):
                    with open(os.path.join(tmp, fname)) as f:
                        extra[suffix] = f.read()
        with open(os.path.join(HERE, "cli", name + ".dat"), "w") as f:
            f.write("# " + args + "\n" + text)
        for suffix, body in extra.items():
            with open(os.path.join(HERE, "cli", name + "." + suffix), "w") as f:
                f.write(body)


# (method mesh, method cao, alpha, uniform, mesh, cao, mc) of the inhomogeneous estimate
INHOMO_CASES = [
    (8, 3, 1.3, 0, 8, 3, 0),
    (8, 3, 1.3, 0, 8, 3, 1),
    (8, 3, 1.3, 0, 8, 5, 1),
    (8, 4, 1.3, 1, 8, 4, 1),
    (16, 2, 1.3, 0, 10, 3, 1),
    (6, 2, 1.3, 0, 6, 2, 2),
    (16, 5, 1.3, 0, 12, 5, 0),
]
# (mesh, cao) of the error map
ERROR_MAP_CASES = [(8, 1), (16, 3), (10, 7), (7, 2)]


def make_inhomo_golden():
    """inhomo.npz: the reference's Generic_error_estimate_inhomo and Error_map
    on a seeded 200-particle system (L = 5), plus the reference's inhomo_output
    columns of case 1."""
    import tempfile
    x, y, z, q = O.uniform_system(200, 5.0, seed=7)
    L = 5.0
    out = dict(x=x, y=y, z=z, q=q, L=L, inhomo_cases=np.array(INHOMO_CASES, dtype=np.float64),
               map_cases=np.array(ERROR_MAP_CASES, dtype=np.float64))
    est = []
    for k, (cm, cc, a, uni, m, c, mc) in enumerate(INHOMO_CASES):
        if k == 1:
            with tempfile.TemporaryDirectory() as tmp:
                f = os.path.join(tmp, "inhomo.txt")
                est.append(O.ref_inhomo_error(x, y, z, q, L, cm, cc, a, uni, m, c, mc, out_file=f))
                out["inhomo_columns_1"] = np.loadtxt(f)
        else:
            est.append(O.ref_inhomo_error(x, y, z, q, L, cm, cc, a, uni, m, c, mc))
    out["inhomo_estimates"] = np.array(est)
    rng = np.random.default_rng(1)
    fk = rng.normal(size=(3, 200))
    fr = fk + 1e-3 * rng.normal(size=(3, 200))
    out["fk"] = fk
    out["fk_ref"] = fr
    for k, (m, c) in enumerate(ERROR_MAP_CASES):
        out["map_%d" % k] = O.ref_error_map(x, y, z, L, fk, fr, m, c)
    np.savez_compressed(os.path.join(HERE, "inhomo.npz"), **out)


# (key, zip archive, position file, exact-force file) from Data/ReferenceDataVincent
VINCENT_FILES = [
    ("nacl300_konfig", "NaCl_crystal_300K.zip", "NaCl_crystal_300K/konfig_0", None),
    ("nacl300", "NaCl_crystal_300K.zip", "NaCl_crystal_300K/Konfig_01.dat", "NaCl_crystal_300K/Konfig_01.exact"),
    ("melt_konfig", "NaCl_melt.zip", "NaCl_melt/konfig_0", None),
    ("melt", "NaCl_melt.zip", "NaCl_melt/Konfig_01.dat", "NaCl_melt/Konfig_01.exact"),
    ("water", "KONFIG_water.zip", "KONFIG_water/CONFIG_water", "KONFIG_water/CONFIG_water.exact"),
]


def make_vincent_golden(ref_dir):
    """vincent.npz: the raw text (uint8 arrays) of the reference's own data
    sets in Data/ReferenceDataVincent: 512-ion NaCl crystal (300 K) and melt
    snapshots in both the konfig_N and the Konfig_NN.dat layout, and the
    648-site water box, with their Konfig_NN.exact / CONFIG_water.exact
    Ewald forces (made outside the reference, by its authors)."""
    import zipfile
    base = os.path.join(ref_dir, "Data", "ReferenceDataVincent")
    out = {}
    for key, arc, pos, exact in VINCENT_FILES:
        with zipfile.ZipFile(os.path.join(base, arc)) as zf:
            out[key + "_pos"] = np.frombuffer(zf.read(pos), dtype=np.uint8)
            if exact:
                out[key + "_exact"] = np.frombuffer(zf.read(exact), dtype=np.uint8)
    np.savez_compressed(os.path.join(HERE, "vincent.npz"), **out)


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
    make_inhomo_golden()
    make_vincent_golden(ref_dir)
    print("wrote", os.path.join(HERE, "wall.npz"), os.path.join(HERE, "sweep.npz"), os.path.join(HERE, "cli"))


def _reference_dir():
    d = os.environ.get("P3M_REFERENCE_DIR")
    if not d:
        sys.exit("give the reference source directory as an argument or in P3M_REFERENCE_DIR")
    return d


if __name__ == "__main__":
    if len(sys.argv) > 2 and sys.argv[1] == "--cli":
        make_cli_goldens(sys.argv[2:])  # only these command-line cases
    elif len(sys.argv) > 1 and sys.argv[1] == "--inhomo":
        make_inhomo_golden()
    elif len(sys.argv) > 1 and sys.argv[1] == "--vincent":
        make_vincent_golden(sys.argv[2] if len(sys.argv) > 2 else _reference_dir())
    else:
        main(sys.argv[1] if len(sys.argv) > 1 else _reference_dir())
