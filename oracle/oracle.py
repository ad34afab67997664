"""ORACLE — test infrastructure only.

ctypes bindings for the CPU oracle restatement (``oracle/liboracle.so``) and
for the reference compiled from its own sources (``oracle/_ref/libp3mref.so``,
present only where ``oracle/build_ref.sh`` ran).  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU legs import this module;
the product path never does.

Force arrays are returned as numpy arrays of shape (3, n) (x, y, z rows),
the reference's SoA layout (types.h:126-132).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def _ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


def _arr(a):
    return np.ascontiguousarray(a, dtype=np.float64)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so missing: run sh oracle/build_oracle.sh")
        L = ctypes.CDLL(path)
        L.oracle_influence.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double, ctypes.c_double, _dp]
        L.oracle_self_force_coeffs.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp]
        L.oracle_kspace.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double, ctypes.c_int] + [_dp] * 4 + [
            ctypes.c_double, _dp, _dp, _dp]
        L.oracle_realspace.argtypes = [ctypes.c_int] + [_dp] * 4 + [ctypes.c_double] * 3 + [_dp, _dp, ctypes.c_int]
        L.oracle_forces.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double, ctypes.c_double, ctypes.c_int] + [
            _dp] * 4 + [ctypes.c_double] + [_dp] * 5 + [ctypes.c_int]
        L.oracle_ewald_parameters.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp, _ip]
        L.oracle_ewald.argtypes = [ctypes.c_int] + [_dp] * 4 + [ctypes.c_double, ctypes.c_int, ctypes.c_int, _ip,
                                                              _dp, _dp, _dp, _dp, _ip]
        L.oracle_ewald_kspace_plain.argtypes = [ctypes.c_int] + [_dp] * 4 + [ctypes.c_double, ctypes.c_double,
                                                                            ctypes.c_int, ctypes.c_int, _ip, _dp]
        L.oracle_rms_error.argtypes = [ctypes.c_int, _dp, _dp]
        L.oracle_rms_error.restype = ctypes.c_double
        L.oracle_realspace_error.argtypes = [ctypes.c_int] + [ctypes.c_double] * 4
        L.oracle_realspace_error.restype = ctypes.c_double
        L.oracle_kspace_error.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                                               ctypes.c_double]
        L.oracle_kspace_error.restype = ctypes.c_double
        L.oracle_bspline.argtypes = [ctypes.c_int, ctypes.c_double, _dp, _dp]
        L.oracle_inhomo_error.argtypes = [ctypes.c_int] + [_dp] * 4 + [ctypes.c_double] * 2 + [ctypes.c_int] * 6 + [
            _dp, _dp]
        L.oracle_error_map.argtypes = [ctypes.c_int] + [_dp] * 3 + [ctypes.c_double, _dp, _dp, ctypes.c_int,
                                                                   ctypes.c_int, _dp]
        _lib = L
    return _lib


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libp3mref.so"))


def ref():
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libp3mref.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/_ref/libp3mref.so missing: run sh oracle/build_ref.sh")
        R = ctypes.CDLL(path)
        R.ref_forces.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double, ctypes.c_double, ctypes.c_int] + [
            _dp] * 4 + [ctypes.c_double] + [_dp] * 5 + [ctypes.c_int, _dp]
        R.ref_self_force_coefficients.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double, ctypes.c_int] + [
            _dp] * 4 + [ctypes.c_double, _dp]
        R.ref_ewald.argtypes = [ctypes.c_int] + [_dp] * 4 + [ctypes.c_double, ctypes.c_int, _dp, _dp, _dp, _dp, _ip]
        R.ref_ewald.restype = ctypes.c_double
        R.ref_error_estimates.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp,
                                                               ctypes.c_double, _dp]
        R.ref_ewald_kspace_main.argtypes = [ctypes.c_int] + [_dp] * 4 + [ctypes.c_double, ctypes.c_int,
                                                                         ctypes.c_double, _dp]
        R.ref_find_error.argtypes = [ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        R.ref_find_error.restype = ctypes.c_double
        R.ref_step_seconds.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double, ctypes.c_double, ctypes.c_int] + [
            _dp] * 4 + [ctypes.c_double, ctypes.c_int]
        R.ref_step_seconds.restype = ctypes.c_double
        R.ref_realteil.argtypes = [ctypes.c_int] + [_dp] * 4 + [ctypes.c_double] * 3 + [_dp, _dp]
        R.ref_inhomo_error.argtypes = [ctypes.c_int] + [_dp] * 4 + [ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                                                    ctypes.c_double] + [ctypes.c_int] * 4 + [
            ctypes.c_char_p]
        R.ref_inhomo_error.restype = ctypes.c_double
        R.ref_error_map.argtypes = [ctypes.c_int] + [_dp] * 3 + [ctypes.c_double, _dp, _dp, ctypes.c_int, ctypes.c_int,
                                                                _dp]
        _ref = R
    return _ref


_refgpu = None


def ref_binding_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libp3mref_gpu.so"))


def ref_binding_forces(gpu, method, mesh, cao, mc, alpha, rcut, x, y, z, q, L, precision=0):
    """The reference's own Init / Influence_function / Calculate_forces
    (common.c:268-327) through its CPU method table (gpu=False) or through
    the p3mg-backed table of p3m-standalone_b200/binding/p3m-gpu.c (gpu=True;
    precision 0 = FP64, 1 = FP32-mixed): dict f, f_k, f_r, energy."""
    global _refgpu
    if _refgpu is None:
        R = ctypes.CDLL(os.path.join(HERE, "_ref", "libp3mref_gpu.so"))
        R.ref_binding_forces.argtypes = [ctypes.c_int] * 6 + [ctypes.c_double, ctypes.c_double, ctypes.c_int] + [
            _dp] * 4 + [ctypes.c_double] + [_dp] * 4
        _refgpu = R
    x, y, z, q = map(_arr, (x, y, z, q))
    n = len(x)
    f, fk, fr, e = np.zeros(3 * n), np.zeros(3 * n), np.zeros(3 * n), np.zeros(1)
    rc = _refgpu.ref_binding_forces(int(bool(gpu)), int(precision), method, mesh, cao, mc, alpha, rcut, n, _ptr(x),
                                    _ptr(y), _ptr(z), _ptr(q), L, _ptr(f), _ptr(fk), _ptr(fr), _ptr(e))
    if rc:
        raise ValueError("ref_binding_forces failed (%d)" % rc)
    return dict(f=f.reshape(3, n), f_k=fk.reshape(3, n), f_r=fr.reshape(3, n), energy=float(e[0]))


def bspline(cao, x):
    w = np.zeros(8)
    dw = np.zeros(8)
    lib().oracle_bspline(cao, x, _ptr(w), _ptr(dw))
    return w[:cao].copy(), dw[:cao].copy()


def influence(method, mesh, cao, mc, alpha, L):
    G = np.zeros(mesh ** 3)
    rc = lib().oracle_influence(method, mesh, cao, mc, alpha, L, _ptr(G))
    if rc:
        raise ValueError("oracle_influence failed (%d)" % rc)
    return G.reshape(mesh, mesh, mesh)


def self_force_coeffs(mesh, cao, L, G):
    G = _arr(G).ravel()
    b = np.zeros(81)
    lib().oracle_self_force_coeffs(mesh, cao, L, _ptr(G), _ptr(b))
    return b


def kspace(method, mesh, cao, mc, alpha, x, y, z, q, L, G=None):
    x, y, z, q = map(_arr, (x, y, z, q))
    n = len(x)
    fk = np.zeros(3 * n)
    ft = np.zeros(3 * n)
    Gp = None if G is None else _arr(G).ravel()
    rc = lib().oracle_kspace(method, mesh, cao, mc, alpha, n, _ptr(x), _ptr(y), _ptr(z), _ptr(q), L, _ptr(Gp),
                             _ptr(fk), _ptr(ft))
    if rc:
        raise ValueError("oracle_kspace failed (%d)" % rc)
    return fk.reshape(3, n), ft.reshape(3, n)


def realspace(x, y, z, q, L, rcut, alpha, cells=True):
    x, y, z, q = map(_arr, (x, y, z, q))
    n = len(x)
    fr = np.zeros(3 * n)
    e = np.zeros(1)
    lib().oracle_realspace(n, _ptr(x), _ptr(y), _ptr(z), _ptr(q), L, rcut, alpha, _ptr(fr), _ptr(e), int(cells))
    return fr.reshape(3, n), float(e[0])


def forces(method, mesh, cao, mc, alpha, rcut, x, y, z, q, L, G=None, cells=True):
    """One Calculate_forces (common.c:268-327): dict with f, f_k, f_r, energy."""
    x, y, z, q = map(_arr, (x, y, z, q))
    n = len(x)
    f = np.zeros(3 * n)
    fk = np.zeros(3 * n)
    fr = np.zeros(3 * n)
    e = np.zeros(1)
    Gp = None if G is None else _arr(G).ravel()
    rc = lib().oracle_forces(method, mesh, cao, mc, alpha, rcut, n, _ptr(x), _ptr(y), _ptr(z), _ptr(q), L,
                             _ptr(Gp), _ptr(f), _ptr(fk), _ptr(fr), _ptr(e), int(cells))
    if rc:
        raise ValueError("oracle_forces failed (%d)" % rc)
    return dict(f=f.reshape(3, n), f_k=fk.reshape(3, n), f_r=fr.reshape(3, n), energy=float(e[0]))


def ewald_parameters(n, q2, L, mesh_param):
    a = np.zeros(1)
    k = np.zeros(1, dtype=np.int32)
    rc = lib().oracle_ewald_parameters(n, q2, L, mesh_param, _ptr(a), k.ctypes.data_as(_ip))
    if rc:
        raise ValueError("Ewald alpha bisection could not start")
    return float(a[0]), int(k[0])


def ewald(x, y, z, q, L, mesh_param, targets=None):
    """FP64 Ewald reference forces (common.c:329-363) on the targets."""
    x, y, z, q = map(_arr, (x, y, z, q))
    n = len(x)
    if targets is None:
        nt, tp, tgt = n, None, None
    else:
        tgt = np.ascontiguousarray(targets, dtype=np.int32)
        nt, tp = len(tgt), tgt.ctypes.data_as(_ip)
    f = np.zeros(3 * nt)
    fk = np.zeros(3 * nt)
    fr = np.zeros(3 * nt)
    a = np.zeros(1)
    k = np.zeros(1, dtype=np.int32)
    rc = lib().oracle_ewald(n, _ptr(x), _ptr(y), _ptr(z), _ptr(q), L, mesh_param, nt, tp, _ptr(f), _ptr(fk),
                            _ptr(fr), _ptr(a), k.ctypes.data_as(_ip))
    if rc:
        raise ValueError("oracle_ewald failed")
    return dict(f=f.reshape(3, nt), f_k=fk.reshape(3, nt), f_r=fr.reshape(3, nt), alpha=float(a[0]), kmax=int(k[0]))


def ewald_kspace_plain(x, y, z, q, L, alpha, kmax, targets=None):
    """Ewald k-space forces with the cutoff 0 < |n|^2 <= kmax^2 (main.c's error_k column uses kmax = mesh - 1)."""
    x, y, z, q = map(_arr, (x, y, z, q))
    n = len(x)
    if targets is None:
        nt, tp = n, None
    else:
        tgt = np.ascontiguousarray(targets, dtype=np.int32)
        nt, tp = len(tgt), tgt.ctypes.data_as(_ip)
    fk = np.zeros(3 * nt)
    lib().oracle_ewald_kspace_plain(n, _ptr(x), _ptr(y), _ptr(z), _ptr(q), L, alpha, kmax, nt, tp, _ptr(fk))
    return fk.reshape(3, nt)


def ref_ewald_kspace_main(x, y, z, q, L, mesh, alpha):
    x, y, z, q = map(_arr, (x, y, z, q))
    fk = np.zeros(3 * len(x))
    ref().ref_ewald_kspace_main(len(x), _ptr(x), _ptr(y), _ptr(z), _ptr(q), L, mesh, alpha, _ptr(fk))
    return fk.reshape(3, len(x))


def kspace_error(method, mesh, cao, mc_est, alpha, n, q2, L):
    return lib().oracle_kspace_error(method, mesh, cao, mc_est, alpha, n, q2, L)


def realspace_error(n, q2, L, rcut, alpha):
    return lib().oracle_realspace_error(n, q2, L, rcut, alpha)


def inhomo_error(x, y, z, q, L, alpha, uniform, mesh, cao, mc, collect_mesh, collect_cao, want_meshes=False):
    """Inhomogeneous k-space error estimate; with want_meshes also the
    (mesh^3, 5) columns rho2, Re E, Im E, Re K2(k), Im K2(k)."""
    x, y, z, q = map(_arr, (x, y, z, q))
    est = np.zeros(1)
    out = np.zeros((mesh ** 3, 5)) if want_meshes else None
    rc = lib().oracle_inhomo_error(len(x), _ptr(x), _ptr(y), _ptr(z), _ptr(q), L, alpha, int(uniform), mesh, cao, mc,
                                   collect_mesh, collect_cao, _ptr(est), _ptr(out))
    if rc:
        raise ValueError("oracle_inhomo_error failed (%d)" % rc)
    return (float(est[0]), out) if want_meshes else float(est[0])


def error_map(x, y, z, L, fk, fk_ref, mesh, cao):
    """Squared k-space force error per particle assigned to a mesh (mesh^3)."""
    x, y, z = map(_arr, (x, y, z))
    fk = _arr(np.asarray(fk).reshape(-1))
    fk_ref = _arr(np.asarray(fk_ref).reshape(-1))
    out = np.zeros(mesh ** 3)
    rc = lib().oracle_error_map(len(x), _ptr(x), _ptr(y), _ptr(z), L, _ptr(fk), _ptr(fk_ref), mesh, cao, _ptr(out))
    if rc:
        raise ValueError("oracle_error_map failed (%d)" % rc)
    return out


# ------------------------------------------------------------ the reference

def ref_forces(method, mesh, cao, mc, alpha, rcut, x, y, z, q, L, tuning=False, want_G=False):
    x, y, z, q = map(_arr, (x, y, z, q))
    n = len(x)
    f = np.zeros(3 * n)
    fk = np.zeros(3 * n)
    fr = np.zeros(3 * n)
    e = np.zeros(1)
    t = np.zeros(3)
    G = np.zeros(mesh ** 3) if want_G else None
    rc = ref().ref_forces(method, mesh, cao, mc, alpha, rcut, n, _ptr(x), _ptr(y), _ptr(z), _ptr(q), L, _ptr(f),
                          _ptr(fk), _ptr(fr), _ptr(G), _ptr(e), int(tuning), _ptr(t))
    if rc:
        raise ValueError("ref_forces failed (%d)" % rc)
    out = dict(f=f.reshape(3, n), f_k=fk.reshape(3, n), f_r=fr.reshape(3, n), energy=float(e[0]), times=t)
    if want_G:
        out["G"] = G.reshape(mesh, mesh, mesh)
    return out


def ref_step_seconds(method, mesh, cao, mc, alpha, rcut, x, y, z, q, L, reps=1):
    """Seconds per Calculate_forces of the reference (its timed region,
    main.c:382-386), the mean of `reps` steps."""
    x, y, z, q = map(_arr, (x, y, z, q))
    t = ref().ref_step_seconds(method, mesh, cao, mc, alpha, rcut, len(x), _ptr(x), _ptr(y), _ptr(z), _ptr(q), L,
                               int(reps))
    if t < 0:
        raise ValueError("ref_step_seconds failed")
    return float(t)


def ref_self_force_coeffs(method, mesh, cao, mc, alpha, x, y, z, q, L):
    x, y, z, q = map(_arr, (x, y, z, q))
    b = np.zeros(81)
    rc = ref().ref_self_force_coefficients(method, mesh, cao, mc, alpha, len(x), _ptr(x), _ptr(y), _ptr(z), _ptr(q),
                                           L, _ptr(b))
    if rc:
        raise ValueError("ref_self_force_coefficients failed")
    return b


def ref_ewald(x, y, z, q, L, mesh_param):
    x, y, z, q = map(_arr, (x, y, z, q))
    n = len(x)
    f = np.zeros(3 * n)
    fk = np.zeros(3 * n)
    fr = np.zeros(3 * n)
    a = np.zeros(1)
    k = np.zeros(1, dtype=np.int32)
    err = ref().ref_ewald(n, _ptr(x), _ptr(y), _ptr(z), _ptr(q), L, mesh_param, _ptr(f), _ptr(fk), _ptr(fr), _ptr(a),
                          k.ctypes.data_as(_ip))
    return dict(f=f.reshape(3, n), f_k=fk.reshape(3, n), f_r=fr.reshape(3, n), alpha=float(a[0]), kmax=int(k[0]),
                err=err)


def ref_error_estimates(method, mesh, cao, mc, alpha, rcut, q, L):
    q = _arr(q)
    e = np.zeros(3)
    rc = ref().ref_error_estimates(method, mesh, cao, mc, alpha, rcut, len(q), _ptr(q), L, _ptr(e))
    if rc:
        raise ValueError("ref_error_estimates failed")
    return e


def ref_find_error(alphaL, mesh, cao, method):
    return ref().ref_find_error(alphaL, mesh, cao, method)


def ref_inhomo_error(x, y, z, q, L, method_mesh, method_cao, alpha, uniform, mesh, cao, mc, out_file=None):
    x, y, z, q = map(_arr, (x, y, z, q))
    return ref().ref_inhomo_error(len(x), _ptr(x), _ptr(y), _ptr(z), _ptr(q), L, method_mesh, method_cao, alpha,
                                  int(uniform), mesh, cao, mc, out_file.encode() if out_file else None)


def ref_error_map(x, y, z, L, fk, fk_ref, mesh, cao):
    x, y, z = map(_arr, (x, y, z))
    fk = _arr(np.asarray(fk).reshape(-1))
    fk_ref = _arr(np.asarray(fk_ref).reshape(-1))
    out = np.zeros(mesh ** 3)
    ref().ref_error_map(len(x), _ptr(x), _ptr(y), _ptr(z), L, _ptr(fk), _ptr(fk_ref), mesh, cao, _ptr(out))
    return out


def estimate_table_mesh(mesh):
    return bool(lib().oracle_estimate_table_mesh(mesh))


def ref_realteil(x, y, z, q, L, rcut, alpha):
    x, y, z, q = map(_arr, (x, y, z, q))
    n = len(x)
    fr = np.zeros(3 * n)
    e = np.zeros(1)
    ref().ref_realteil(n, _ptr(x), _ptr(y), _ptr(z), _ptr(q), L, rcut, alpha, _ptr(fr), _ptr(e))
    return fr.reshape(3, n), float(e[0])


def rel_rms(a, b):
    """sqrt(sum |a-b|^2) / sqrt(sum |b|^2) over all components."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.sqrt(np.sum(b * b))
    return float(np.sqrt(np.sum((a - b) ** 2)) / den) if den > 0 else float(np.sqrt(np.sum((a - b) ** 2)))


def abs_rms(a, b):
    """sqrt(sum_i |a_i - b_i|^2 / n) for (3, n) arrays (error.c:21-34)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.sqrt(np.sum((a - b) ** 2) / a.shape[-1]))


def uniform_system(n, L, seed=12345):
    """Seeded uniform system, charges (1 - 2 (i mod 2)) as in generate_system.c:162."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, L, size=(3, n))
    pos = np.where(pos >= L, 0.0, pos)
    q = 1.0 - 2.0 * (np.arange(n) % 2)
    return pos[0].copy(), pos[1].copy(), pos[2].copy(), q
