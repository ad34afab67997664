"""Python host side of p3mg: ctypes bindings over the C ABI (include/p3mg.h)
and a mirror of the reference's plugin interface for the P3M force path.

The reference selects a ``method_t`` by numeric id (main.c:314-344) and
drives it as Init -> Influence_function (per alpha) -> Calculate_forces
(common.c:268-327).  ``Method`` below keeps those names, ids and the
accumulate-into semantics; ``calculate_forces`` is Calculate_forces.  The
compute runs in ``libp3mg.so`` (hand-written sm_100a kernels); there is no
CPU fallback -- loading fails loudly when the library or a GPU is missing.

Arrays: positions, charges and forces are numpy float64; forces are (3, n)
arrays (the reference's SoA vector_array_t, types.h:126-132).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

OK = 0
# status codes of include/p3mg.h
ERR_ARG, ERR_METHOD, ERR_CAO, ERR_MESH, ERR_NOSYS = -1, -2, -3, -4, -5
ERR_CUDA, ERR_ALLOC, ERR_STATE, ERR_PRECISION, ERR_NOBUF = -6, -7, -8, -9, -10
FP64 = 0
FP32_MIXED = 1

# method ids and names of the reference's method_t tables
METHODS = {
    0: ("P3M with ik differentiation, not intelaced.", "p3m-ik"),
    1: ("P3M with ik differentiation, interlaced.", "p3m-ik-i"),
    2: ("P3M with analytic differentiation, not intelaced.", "p3m-ad"),
    3: ("P3M with analytic differentiation, intelaced.", "p3m-ad-i"),
    6: ("P3M with ik differentiation, not intelaced, real input.", "p3m-ik-r"),
    7: ("P3M with analytic differentiation, not intelaced, real input.", "p3m-ad-r"),
}

# method_t flags (types.h:290-303)
FLAG_IK, FLAG_AD, FLAG_INTERLACED, FLAG_SELF_FORCE = 1, 2, 4, 128
METHOD_FLAGS = {
    0: FLAG_IK, 1: FLAG_IK | FLAG_INTERLACED, 2: FLAG_AD | FLAG_SELF_FORCE, 3: FLAG_AD | FLAG_INTERLACED,
    6: FLAG_IK, 7: FLAG_AD | FLAG_SELF_FORCE,
}


class P3MGError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = _lib_or_none().p3mg_strerror(status).decode() if _lib_or_none() else str(status)
        extra = ""
        if status == -6 and _lib_or_none():
            extra = " (%s)" % _lib_or_none().p3mg_last_cuda_error().decode()
        super().__init__("%s: %s [status %d]%s" % (what, msg, status, extra))


_dp = ctypes.POINTER(ctypes.c_double)
_LIB = None


def _lib_or_none():
    return _LIB


def lib_path():
    return os.path.join(HERE, "libp3mg.so")


def load():
    """Load libp3mg.so (built by p3m-standalone_b200/build.py).  Raises if absent."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not os.path.exists(path):
        raise RuntimeError("libp3mg.so not found at %s: run python p3m-standalone_b200/build.py" % path)
    L = ctypes.CDLL(path)
    vp = ctypes.c_void_p
    L.p3mg_create.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.c_int]
    L.p3mg_destroy.argtypes = [vp]
    L.p3mg_destroy.restype = None
    L.p3mg_set_system.argtypes = [vp, ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_double]
    L.p3mg_set_system_device.argtypes = [vp, ctypes.c_int, vp, vp, vp, vp, ctypes.c_double]
    L.p3mg_influence.argtypes = [vp, ctypes.c_double]
    L.p3mg_kspace_forces.argtypes = [vp] + [_dp] * 6
    L.p3mg_real_forces.argtypes = [vp, ctypes.c_double, ctypes.c_double] + [_dp] * 4
    L.p3mg_calculate_forces.argtypes = [vp, ctypes.c_double] + [_dp] * 10
    L.p3mg_compute.argtypes = [vp, ctypes.c_double]
    L.p3mg_get_forces.argtypes = [vp] + [_dp] * 10
    L.p3mg_get_forces_device.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp)]
    L.p3mg_enable_timing.argtypes = [vp, ctypes.c_int]
    L.p3mg_stage_times.argtypes = [vp, _dp]
    L.p3mg_get_influence.argtypes = [vp, _dp, _dp]
    L.p3mg_ewald_forces.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), _dp, _dp, _dp, _dp,
                                    ctypes.POINTER(ctypes.c_int)]
    L.p3mg_ewald_reference.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)] + [_dp] * 7 + [
        ctypes.POINTER(ctypes.c_int), _dp]
    L.p3mg_ewald_kspace_forces.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                           ctypes.POINTER(ctypes.c_int), _dp, _dp, _dp]
    L.p3mg_alpha_range.argtypes = [ctypes.c_double] * 3 + [ctypes.c_int, _dp]
    L.p3mg_sweep.argtypes = [vp, ctypes.c_double, ctypes.c_int, _dp, _dp, _dp, _dp, _dp, _dp, ctypes.c_int]
    L.p3mg_sweep_nodes.argtypes = [vp, ctypes.POINTER(ctypes.c_int), _dp]
    L.p3mg_sweep_grid.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp, _dp, _dp,
                                  _dp, _dp]
    L.p3mg_energy.argtypes = [vp, ctypes.c_double, _dp]
    L.p3mg_backward.argtypes = [vp, ctypes.c_double, ctypes.c_double] + [_dp] * 7
    L.p3mg_backward_device.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.POINTER(vp),
                                       ctypes.POINTER(vp), _dp, _dp, _dp]
    L.p3mg_set_tiles.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    L.p3mg_set_gather.argtypes = [vp, ctypes.c_int]
    _ip = ctypes.POINTER(ctypes.c_int)
    L.p3mg_autotune.argtypes = [vp, ctypes.c_double, _ip, _ip, _dp]
    L.p3mg_tune.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int] + [_dp] * 4 + [ctypes.c_double] * 3 + [
        ctypes.c_int, ctypes.c_int, _ip, _ip, _dp, _dp, _dp]
    L.p3mg_batch_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.c_int]
    L.p3mg_batch_compute.argtypes = [vp, _dp]
    L.p3mg_batch_synchronize.argtypes = [vp]
    L.p3mg_batch_destroy.argtypes = [vp]
    L.p3mg_batch_destroy.restype = None
    L.p3mg_estimate_errors.argtypes = [ctypes.c_int] * 5 + [ctypes.c_double] * 4 + [_dp]
    L.p3mg_error_estimate.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp]
    L.p3mg_inhomo_error.argtypes = [vp, ctypes.c_double] + [ctypes.c_int] * 6 + [_dp, _dp]
    L.p3mg_error_map.argtypes = [vp, ctypes.c_int, ctypes.c_int] + [_dp] * 8
    L.p3mg_kernel_times.argtypes = [vp, _dp]
    L.p3mg_set_graph.argtypes = [vp, ctypes.c_int]
    L.p3mg_set_overlap.argtypes = [vp, ctypes.c_int]
    L.p3mg_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong)]
    L.p3mg_stream.argtypes = [vp]
    L.p3mg_stream.restype = vp
    L.p3mg_strerror.argtypes = [ctypes.c_int]
    L.p3mg_strerror.restype = ctypes.c_char_p
    L.p3mg_last_cuda_error.argtypes = []
    L.p3mg_last_cuda_error.restype = ctypes.c_char_p
    _LIB = L
    return L


def _check(status, what):
    if status != OK:
        raise P3MGError(status, what)


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Context:
    """One p3mg context: a method on one mesh, owning its device memory."""

    def __init__(self, method, mesh, cao, mc=1, precision=FP64):
        self._lib = load()
        self._h = ctypes.c_void_p()
        _check(self._lib.p3mg_create(ctypes.byref(self._h), int(method), int(mesh), int(cao), int(mc),
                                     int(precision)), "p3mg_create")
        self.method, self.mesh, self.cao, self.mc, self.precision = method, mesh, cao, mc, precision
        self.n = 0
        self.L = None

    def close(self):
        if self._h:
            self._lib.p3mg_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def handle(self):
        return self._h

    def set_system(self, x, y, z, q, L):
        x, y, z, q = map(_f64, (x, y, z, q))
        self._keep = (x, y, z, q)
        _check(self._lib.p3mg_set_system(self._h, len(x), _p(x), _p(y), _p(z), _p(q), float(L)), "p3mg_set_system")
        self.n, self.L = len(x), float(L)

    def set_system_device(self, n, px, py, pz, pq, L):
        """Device pointers (ints) to n doubles each."""
        _check(self._lib.p3mg_set_system_device(self._h, int(n), ctypes.c_void_p(px), ctypes.c_void_p(py),
                                                ctypes.c_void_p(pz), ctypes.c_void_p(pq), float(L)),
               "p3mg_set_system_device")
        self.n, self.L = int(n), float(L)

    def influence(self, alpha):
        _check(self._lib.p3mg_influence(self._h, float(alpha)), "p3mg_influence")

    def kspace_forces(self, fk=None, ftot=None):
        n = self.n
        fk = np.zeros((3, n)) if fk is None else fk
        args = [_p(fk[0]), _p(fk[1]), _p(fk[2])]
        args += [None] * 3 if ftot is None else [_p(ftot[0]), _p(ftot[1]), _p(ftot[2])]
        _check(self._lib.p3mg_kspace_forces(self._h, *args), "p3mg_kspace_forces")
        return fk

    def real_forces(self, rcut, alpha, fr=None):
        n = self.n
        fr = np.zeros((3, n)) if fr is None else fr
        e = ctypes.c_double(0.0)
        _check(self._lib.p3mg_real_forces(self._h, float(rcut), float(alpha), _p(fr[0]), _p(fr[1]), _p(fr[2]),
                                          ctypes.byref(e)), "p3mg_real_forces")
        return fr, e.value

    def calculate_forces(self, rcut):
        """Calculate_forces (common.c:268-327): dict f, f_k, f_r, energy."""
        n = self.n
        f, fk, fr = np.zeros((3, n)), np.zeros((3, n)), np.zeros((3, n))
        e = ctypes.c_double(0.0)
        _check(self._lib.p3mg_calculate_forces(self._h, float(rcut), _p(f[0]), _p(f[1]), _p(f[2]), _p(fk[0]),
                                               _p(fk[1]), _p(fk[2]), _p(fr[0]), _p(fr[1]), _p(fr[2]),
                                               ctypes.byref(e)), "p3mg_calculate_forces")
        return dict(f=f, f_k=fk, f_r=fr, energy=e.value)

    def compute(self, rcut):
        _check(self._lib.p3mg_compute(self._h, float(rcut)), "p3mg_compute")

    def get_forces(self):
        n = self.n
        f, fk, fr = np.zeros((3, n)), np.zeros((3, n)), np.zeros((3, n))
        e = ctypes.c_double(0.0)
        _check(self._lib.p3mg_get_forces(self._h, _p(f[0]), _p(f[1]), _p(f[2]), _p(fk[0]), _p(fk[1]), _p(fk[2]),
                                         _p(fr[0]), _p(fr[1]), _p(fr[2]), ctypes.byref(e)), "p3mg_get_forces")
        return dict(f=f, f_k=fk, f_r=fr, energy=e.value)

    def forces_device(self):
        """Device pointers (ints) to the f, f_k, f_r arrays (3n doubles each)."""
        a, b, c = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        _check(self._lib.p3mg_get_forces_device(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)),
               "p3mg_get_forces_device")
        return a.value, b.value, c.value

    def enable_timing(self, on=True):
        _check(self._lib.p3mg_enable_timing(self._h, int(bool(on))), "p3mg_enable_timing")

    def stage_times(self):
        t = np.zeros(4)
        _check(self._lib.p3mg_stage_times(self._h, _p(t)), "p3mg_stage_times")
        return dict(t_c=t[0], t_g=t[1], t_f=t[2], t_r=t[3])

    def _targets(self, targets):
        if targets is None:
            return self.n, None
        tg = np.ascontiguousarray(targets, dtype=np.int32)
        self._tg = tg
        return len(tg), tg.ctypes.data_as(ctypes.POINTER(ctypes.c_int))

    def ewald_forces(self, targets=None):
        """FP64 Ewald reference forces on the targets (indices; None = all):
        dict f (3, nt), alpha, kmax (Calculate_reference_forces, common.c:329-363)."""
        nt, tp = self._targets(targets)
        f = np.zeros((3, nt))
        a = ctypes.c_double(0.0)
        k = ctypes.c_int(0)
        _check(self._lib.p3mg_ewald_forces(self._h, nt, tp, _p(f[0]), _p(f[1]), _p(f[2]), ctypes.byref(a),
                                           ctypes.byref(k)), "p3mg_ewald_forces")
        return dict(f=f, alpha=a.value, kmax=k.value)

    def ewald_reference(self, targets=None):
        """Every output of Calculate_reference_forces: dict f, f_k (3, nt), alpha,
        kmax and the Ewald error estimate 'precision'."""
        nt, tp = self._targets(targets)
        f = np.zeros((3, nt))
        fk = np.zeros((3, nt))
        a = ctypes.c_double(0.0)
        k = ctypes.c_int(0)
        e = ctypes.c_double(0.0)
        _check(self._lib.p3mg_ewald_reference(self._h, nt, tp, _p(f[0]), _p(f[1]), _p(f[2]), _p(fk[0]), _p(fk[1]),
                                              _p(fk[2]), ctypes.byref(a), ctypes.byref(k), ctypes.byref(e)),
               "p3mg_ewald_reference")
        return dict(f=f, f_k=fk, alpha=a.value, kmax=k.value, precision=e.value)

    def ewald_kspace_forces(self, alpha, kmax, targets=None):
        """Ewald k-space forces (3, nt) with the cutoff 0 < |n|^2 <= kmax^2."""
        nt, tp = self._targets(targets)
        fk = np.zeros((3, nt))
        _check(self._lib.p3mg_ewald_kspace_forces(self._h, float(alpha), int(kmax), nt, tp, _p(fk[0]), _p(fk[1]),
                                                  _p(fk[2])), "p3mg_ewald_kspace_forces")
        return fk

    def sweep(self, rcut, alphas, ref=None, want_forces=False, max_batch=0):
        """Batched alpha sweep (p3mg_sweep): dict rms (per alpha, when ref (3, n)
        is given) and forces (nalpha, 3, n) when want_forces; nodes (> 0: the
        forces were interpolated from that many Chebyshev nodes in 1/alpha^2)
        and check.  max_batch 0 lets a wide enough sweep interpolate; max_batch
        > 0 evaluates every alpha, at most max_batch of them in one pass."""
        al = np.ascontiguousarray(alphas, dtype=np.float64)
        na = len(al)
        rms = np.zeros(na) if ref is not None else None
        f = np.zeros((na, 3, self.n)) if want_forces else None
        if ref is not None:
            r = np.ascontiguousarray(ref, dtype=np.float64).reshape(3, self.n)
            rx, ry, rz = (np.ascontiguousarray(r[d]) for d in range(3))
        else:
            rx = ry = rz = None
        _check(self._lib.p3mg_sweep(self._h, float(rcut), na, _p(al), _p(rx), _p(ry), _p(rz), _p(rms), _p(f),
                                    int(max_batch)), "p3mg_sweep")
        nodes = ctypes.c_int(0)
        check = np.zeros(1)
        _check(self._lib.p3mg_sweep_nodes(self._h, ctypes.byref(nodes), _p(check)), "p3mg_sweep_nodes")
        return dict(rms=rms, forces=f, nodes=nodes.value, check=float(check[0]))

    def energy(self, rcut):
        """P3M energy parts (p3mg_energy): dict total, kspace, realspace, self, neutral."""
        e = np.zeros(5)
        _check(self._lib.p3mg_energy(self._h, float(rcut), _p(e)), "p3mg_energy")
        return dict(zip(("total", "kspace", "realspace", "self", "neutral"), e))

    def backward(self, rcut, grad_E=1.0):
        """Adjoint (p3mg_backward): dict energy (parts), dx (3, n), dq (n), dalpha, dL,
        each grad_E times the derivative of the total energy."""
        n = self.n
        gx, gq, e = np.zeros((3, n)), np.zeros(n), np.zeros(5)
        da, dl = np.zeros(1), np.zeros(1)
        _check(self._lib.p3mg_backward(self._h, float(rcut), float(grad_E), _p(gx[0]), _p(gx[1]), _p(gx[2]),
                                       _p(gq), _p(da), _p(dl), _p(e)), "p3mg_backward")
        return dict(energy=dict(zip(("total", "kspace", "realspace", "self", "neutral"), e)), dx=gx, dq=gq,
                    dalpha=float(da[0]), dL=float(dl[0]))

    def backward_device(self, rcut, grad_E=1.0):
        """p3mg_backward_device: dict energy parts, dalpha, dL and the device
        pointers (ints) of the gradients dx (3n) and dq (n)."""
        gx, gq = ctypes.c_void_p(), ctypes.c_void_p()
        da, dl, e5 = ctypes.c_double(0.0), ctypes.c_double(0.0), np.zeros(5)
        _check(self._lib.p3mg_backward_device(self._h, float(rcut), float(grad_E), ctypes.byref(gx), ctypes.byref(gq),
                                              ctypes.byref(da), ctypes.byref(dl), _p(e5)), "p3mg_backward_device")
        return dict(energy=dict(zip(("total", "kspace", "realspace", "self", "neutral"), e5)), dalpha=da.value,
                    dL=dl.value, dx_ptr=gx.value, dq_ptr=gq.value)

    def set_tiles(self, brick, fft_w=0):
        _check(self._lib.p3mg_set_tiles(self._h, int(brick), int(fft_w)), "p3mg_set_tiles")

    def set_gather(self, mode):
        """ik back-interpolation kernel: 0 lanes on the stencil's z offsets, 1 one thread per particle,
        2 (FP32) TMA-staged brick tiles in shared memory, 3 (FP32) the same tiles with plain loads."""
        _check(self._lib.p3mg_set_gather(self._h, int(mode)), "p3mg_set_gather")

    def autotune(self, rcut):
        """Tile autotuner (p3mg_autotune): dict brick, fft_w, ms."""
        b, w, t = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0.0)
        _check(self._lib.p3mg_autotune(self._h, float(rcut), ctypes.byref(b), ctypes.byref(w), ctypes.byref(t)),
               "p3mg_autotune")
        return dict(brick=b.value, fft_w=w.value, ms=t.value)

    def error_estimate(self, alpha, rcut, mc_est=1):
        """Analytic RMS error estimates (method.Error / Error_k, Realspace_error):
        dict total, kspace, realspace."""
        e = np.zeros(3)
        _check(self._lib.p3mg_error_estimate(self._h, float(alpha), float(rcut), int(mc_est), _p(e)),
               "p3mg_error_estimate")
        return dict(total=e[0], kspace=e[1], realspace=e[2])

    def inhomo_error(self, alpha, mesh=64, cao=5, mc=0, uniform=False, collect_mesh=None, collect_cao=None,
                     want_meshes=False):
        """Inhomogeneous k-space error estimate (p3mg_inhomo_error).  collect_mesh /
        collect_cao default to the estimator's mesh and cao (the reference's CLI
        passes the force method's).  With want_meshes also the (mesh^3, 5) columns
        rho2, Re E, Im E, Re DFT(K2), Im DFT(K2)."""
        cm = mesh if collect_mesh is None else collect_mesh
        cc = cao if collect_cao is None else collect_cao
        est = np.zeros(1)
        out = np.zeros((mesh ** 3, 5)) if want_meshes else None
        _check(self._lib.p3mg_inhomo_error(self._h, float(alpha), int(bool(uniform)), int(mesh), int(cao), int(mc),
                                           int(cm), int(cc), _p(est), _p(out)), "p3mg_inhomo_error")
        return (float(est[0]), out) if want_meshes else float(est[0])

    def error_map(self, fk, ref, mesh=64, cao=1):
        """Error map (p3mg_error_map): (mesh^3 doubles, totals (2,)) for k-space
        forces fk and reference forces ref, both (3, n)."""
        fk = np.ascontiguousarray(fk, dtype=np.float64).reshape(3, self.n)
        ref = np.ascontiguousarray(ref, dtype=np.float64).reshape(3, self.n)
        a = [np.ascontiguousarray(fk[d]) for d in range(3)] + [np.ascontiguousarray(ref[d]) for d in range(3)]
        out = np.zeros(mesh ** 3)
        tot = np.zeros(2)
        _check(self._lib.p3mg_error_map(self._h, int(mesh), int(cao), *[_p(v) for v in a], _p(out), _p(tot)),
               "p3mg_error_map")
        return out, tot

    def kernel_times(self):
        t = np.zeros(3)
        _check(self._lib.p3mg_kernel_times(self._h, _p(t)), "p3mg_kernel_times")
        return dict(pairs=t[0], scatter=t[1], gather=t[2])

    def set_graph(self, on=True):
        _check(self._lib.p3mg_set_graph(self._h, int(bool(on))), "p3mg_set_graph")

    def set_overlap(self, on=True):
        """Real-space pairs beside the k-space chain (True, the default) or before it."""
        _check(self._lib.p3mg_set_overlap(self._h, int(bool(on))), "p3mg_set_overlap")

    def launch_count(self):
        c = ctypes.c_longlong(0)
        _check(self._lib.p3mg_launch_count(self._h, ctypes.byref(c)), "p3mg_launch_count")
        return int(c.value)

    def set_system_ptr(self, n, px, py, pz, pq, L):
        """Host pointers (ints, e.g. pinned torch tensors) to n doubles each."""
        P = lambda v: ctypes.cast(ctypes.c_void_p(v), _dp)  # noqa: E731
        _check(self._lib.p3mg_set_system(self._h, int(n), P(px), P(py), P(pz), P(pq), float(L)), "p3mg_set_system")
        self.n, self.L = int(n), float(L)

    def get_total_forces_ptr(self, px, py, pz):
        """Copy the total force of the last compute to host pointers (ints)."""
        P = lambda v: ctypes.cast(ctypes.c_void_p(v), _dp)  # noqa: E731
        _check(self._lib.p3mg_get_forces(self._h, P(px), P(py), P(pz), None, None, None, None, None, None, None),
               "p3mg_get_forces")

    def get_influence(self):
        G = np.zeros(self.mesh ** 3)
        b = np.zeros(81)
        _check(self._lib.p3mg_get_influence(self._h, _p(G), _p(b)), "p3mg_get_influence")
        return G.reshape(self.mesh, self.mesh, self.mesh), b

    def stream(self):
        return self._lib.p3mg_stream(self._h)


class Method:
    """Mirror of the reference's method_t (types.h:306-316) for one id.

    Init -> Context; Influence_function(alpha); Kspace_force accumulates into
    forces['f_k'] (and subtracts the ad self-force from forces['f']).
    """

    def __init__(self, method_id):
        if method_id not in METHODS:
            raise P3MGError(-2, "method %r" % (method_id,)) if _LIB else ValueError("method %r not known" % method_id)
        self.method_id = method_id
        self.method_name, self.method_name_short = METHODS[method_id]
        self.flags = METHOD_FLAGS[method_id]

    def Init(self, x, y, z, q, L, mesh, cao, mc=1, precision=FP64):
        ctx = Context(self.method_id, mesh, cao, mc, precision)
        ctx.set_system(x, y, z, q, L)
        return ctx

    @staticmethod
    def Influence_function(ctx, alpha):
        ctx.influence(alpha)

    @staticmethod
    def Kspace_force(ctx, forces):
        ctx.kspace_forces(forces["f_k"], forces["f"])


def sweep_grid(contexts, rcut, alphas, ref):
    """p3mg_sweep_grid: RMS error against ref (3, n) of every context (same
    system, different mesh / cao / method) at every alpha, real space
    shared; returns an array (len(contexts), len(alphas))."""
    alphas = np.ascontiguousarray(alphas, dtype=np.float64)
    ref = np.ascontiguousarray(ref, dtype=np.float64)
    hs = (ctypes.c_void_p * len(contexts))(*[c.handle.value for c in contexts])
    out = np.zeros((len(contexts), len(alphas)))
    _check(load().p3mg_sweep_grid(hs, len(contexts), float(rcut), len(alphas), _p(alphas), _p(ref[0]), _p(ref[1]),
                                  _p(ref[2]), _p(out)), "p3mg_sweep_grid")
    return out


def alpha_range(alphamin, alphamax, alphastep):
    """The reference sweep's alphas (p3mg_alpha_range, main.c:375)."""
    L = load()
    k = L.p3mg_alpha_range(float(alphamin), float(alphamax), float(alphastep), 0, None)
    if k < 0:
        raise P3MGError(k, "p3mg_alpha_range")
    out = np.zeros(k)
    L.p3mg_alpha_range(float(alphamin), float(alphamax), float(alphastep), k, _p(out))
    return out


class Batch:
    """Several contexts' force evaluations as one CUDA graph (p3mg_batch_*)."""

    def __init__(self, contexts):
        self._lib = load()
        self.contexts = list(contexts)
        arr = (ctypes.c_void_p * len(self.contexts))(*[c._h.value for c in self.contexts])
        self._h = ctypes.c_void_p(0)
        _check(self._lib.p3mg_batch_create(ctypes.byref(self._h), arr, len(self.contexts)), "p3mg_batch_create")

    def compute(self, rcuts):
        r = np.ascontiguousarray(np.broadcast_to(np.asarray(rcuts, dtype=np.float64), (len(self.contexts),)))
        _check(self._lib.p3mg_batch_compute(self._h, _p(r)), "p3mg_batch_compute")

    def synchronize(self):
        _check(self._lib.p3mg_batch_synchronize(self._h), "p3mg_batch_synchronize")

    def close(self):
        if self._h:
            self._lib.p3mg_batch_destroy(self._h)
            self._h = ctypes.c_void_p(0)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def tune(method, x, y, z, q, L, rcut, target, precision=FP64, cao=0, mesh_max=0):
    """The reference's Tune on the GPU (p3mg_tune): dict mesh, cao, alpha, estimate, ms."""
    x, y, z, q = (np.ascontiguousarray(v, dtype=np.float64) for v in (x, y, z, q))
    m, c = ctypes.c_int(0), ctypes.c_int(0)
    a, e, t = ctypes.c_double(0.0), ctypes.c_double(0.0), ctypes.c_double(0.0)
    _check(load().p3mg_tune(int(method), int(precision), len(x), _p(x), _p(y), _p(z), _p(q), float(L), float(rcut),
                            float(target), int(cao), int(mesh_max), ctypes.byref(m), ctypes.byref(c), ctypes.byref(a),
                            ctypes.byref(e), ctypes.byref(t)), "p3mg_tune")
    return dict(mesh=m.value, cao=c.value, alpha=a.value, estimate=e.value, ms=t.value)


def estimate_errors(method, mesh, cao, n, q2, L, alpha, rcut, mc_est=1):
    """Analytic RMS error estimates without a context (p3mg_estimate_errors):
    dict total, kspace, realspace."""
    e = np.zeros(3)
    _check(load().p3mg_estimate_errors(int(method), int(mesh), int(cao), int(mc_est), int(n), float(q2), float(L),
                                       float(alpha), float(rcut), _p(e)), "p3mg_estimate_errors")
    return dict(total=e[0], kspace=e[1], realspace=e[2])


def calculate_forces(ctx, rcut):
    """Calculate_forces (common.c:268-327) on a context with G computed."""
    return ctx.calculate_forces(rcut)


# ------------------------------------------------------------------ systems

SYSTEM_RANDOM, SYSTEM_INNER_BOX, SYSTEM_MADELUNG, SYSTEM_SEPARATED_DIPOLE, SYSTEM_GAUSSIAN, SYSTEM_SLAB = range(6)


def generate_system(system_type, n, L, charge=1.0, seed=12345, sigma=None):
    """Seeded synthetic systems of the reference's types (generate_system.c,
    README 'system_type'): returns x, y, z, q (float64) with positions in
    [0, L).  The generator is numpy's PCG64, not GSL's stream; inputs are
    shared with the reference through the position-file format.

    0 uniform; 1 inner box [0.25L, 0.75L)^3; 2 Madelung crystal; 3 separated
    dipoles (pairs at distance 1, isotropic); 4 Gaussian about the centre
    (sigma default L/6, rejection to [0, L)); 5 slab x in [0.25L, 0.75L)
    (README:57 geometry)."""
    rng = np.random.default_rng(seed)
    alt = 1.0 - 2.0 * (np.arange(n) % 2)
    if system_type == SYSTEM_RANDOM:
        p = rng.uniform(0.0, L, size=(3, n))
        q = alt * charge
    elif system_type == SYSTEM_INNER_BOX:
        p = 0.25 * L + 0.5 * L * rng.uniform(0.0, 1.0, size=(3, n))
        q = alt.copy()
    elif system_type == SYSTEM_MADELUNG:
        per_row = int(np.ceil(n ** (1.0 / 3.0) - 1e-9))
        a = L / per_row
        i, j, k = np.meshgrid(np.arange(per_row), np.arange(per_row), np.arange(per_row), indexing="ij")
        p = np.stack([a * i.ravel() + 0.5 * a, a * j.ravel() + 0.5 * a, a * k.ravel() + 0.5 * a])
        q = 1.0 - 2.0 * ((i + j + k).ravel() % 2)
    elif system_type == SYSTEM_SEPARATED_DIPOLE:
        nd = n // 2
        c = L * rng.uniform(0.0, 1.0, size=(3, nd))
        u = rng.uniform(-1.0, 1.0, size=nd)
        th = 2.0 * np.pi * rng.uniform(0.0, 1.0, size=nd)
        s = np.sqrt(1.0 - u * u)
        d = np.stack([s * np.cos(th), s * np.sin(th), u])
        p = np.empty((3, 2 * nd))
        p[:, 0::2] = c
        p[:, 1::2] = np.mod(c + d, L)
        q = np.empty(2 * nd)
        q[0::2] = 1.0
        q[1::2] = -1.0
    elif system_type == SYSTEM_GAUSSIAN:
        sig = L / 6.0 if sigma is None else sigma
        p = np.empty((3, n))
        for dim in range(3):
            v = rng.normal(L / 2.0, sig, size=n)
            bad = (v < 0.0) | (v >= L)
            while bad.any():
                v[bad] = rng.normal(L / 2.0, sig, size=int(bad.sum()))
                bad = (v < 0.0) | (v >= L)
            p[dim] = v
        q = alt * charge
    elif system_type == SYSTEM_SLAB:
        p = rng.uniform(0.0, L, size=(3, n))
        p[0] = 0.25 * L + 0.5 * L * rng.uniform(0.0, 1.0, size=n)
        q = alt.copy()
    else:
        raise ValueError("system_type %r not known" % (system_type,))
    p = np.where(p >= L, p - L, p)
    return p[0].copy(), p[1].copy(), p[2].copy(), np.asarray(q, dtype=np.float64)


# --------------------------------------------------------------- file formats

def read_system(path):
    """Read_system (io.c:100-157): '# Teilchenzahl: N', '# Len: L', then
    N lines 'x y z q'.  Extra '#' header lines (the '# Mesh:', '# kmax:',
    '# alpha:' ... lines of the Data/ReferenceDataVincent Konfig_NN.dat
    files, see read_system_header) are skipped.  A file without the '#'
    header is a konfig_N simulation snapshot of the same data sets: a count
    line, a box-length line, then 'x y z q' with unwrapped coordinates,
    which are folded into [0, L)."""
    with open(path) as fh:
        lines = [l.strip() for l in fh]
    lines = [l for l in lines if l]
    if not lines:
        raise ValueError("Error while reading file '%s'" % path)
    if not lines[0].startswith("#"):
        try:
            n, L = int(lines[0].split()[0]), float(lines[1].split()[0])
            a = np.array([[float(v) for v in l.split()[:4]] for l in lines[2:2 + n]], dtype=np.float64).reshape(-1, 4)
        except (ValueError, IndexError):
            raise ValueError("Error while reading file '%s'" % path)
        if a.shape[0] != n or not L > 0:
            raise ValueError("Error while reading file '%s': %d of %d particles" % (path, a.shape[0], n))
        pos = a[:, :3] - L * np.floor(a[:, :3] / L)
        pos[(pos >= L) | (pos < 0)] = 0.0
        return pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(), a[:, 3].copy(), L
    hdr = read_system_header(path)
    n, L = hdr.get("Teilchenzahl"), hdr.get("Len")
    if n is None or L is None:
        raise ValueError("Error while reading file '%s'" % path)
    n = int(n)
    rows = []
    for l in lines:
        if l.startswith("#"):
            continue
        rows.append([float(v) for v in l.split()[:4]])
        if len(rows) == n:
            break
    a = np.array(rows, dtype=np.float64).reshape(-1, 4)
    if a.shape[0] != n:
        raise ValueError("Error while reading file '%s': %d of %d particles" % (path, a.shape[0], n))
    return a[:, 0].copy(), a[:, 1].copy(), a[:, 2].copy(), a[:, 3].copy(), float(L)


def read_system_header(path):
    """The '# key: value' header lines of a positions file as a dict of
    numbers: Teilchenzahl and Len, and in the Konfig_NN.dat files of
    Data/ReferenceDataVincent also Mesh, kmax, alpha, beta, ip (the window
    order minus 1), rcut, Temp and Bjerrum."""
    out = {}
    with open(path) as fh:
        for line in fh:
            s = line.strip()
            if not s:
                continue
            if not s.startswith("#"):
                break
            key, _, val = s[1:].partition(":")
            try:
                v = float(val)
            except ValueError:
                continue
            out[key.strip()] = int(v) if v.is_integer() and key.strip() in ("Teilchenzahl", "Mesh", "kmax", "ip") \
                else v
    return out


def write_system(path, x, y, z, q, L):
    """Write_system (io.c:199-225), same '%lf' text format."""
    with open(path, "w") as fh:
        fh.write("# Teilchenzahl: %d\n" % len(x))
        fh.write("# Len: %f\n" % L)
        for i in range(len(x)):
            fh.write("%f\t%f\t%f\t%f\n" % (x[i], y[i], z[i], q[i]))


def read_exact_forces(path, n, with_energy=False):
    """Read_exact_forces (io.c:70-98): lines 'id fx fy fz'.  Also accepts the
    7-column 'id F(3) F_k(3)' layout Write_exact_forces writes (io.c:171-173),
    taking the total force columns, and the Konfig_NN.exact lines
    'E fx fy fz' of Data/ReferenceDataVincent (first field not an integer:
    the total Coulomb energy).  with_energy: also return that energy (None
    for the other layouts)."""
    f = np.zeros((3, n))
    energy = None
    i = 0
    with open(path) as fh:
        for line in fh:
            s = line.split()
            if not s:
                continue
            integer = not any(c in s[0] for c in ".eE")
            if len(s) not in (4, 7) or (len(s) == 7 and not integer):
                raise ValueError("Error while reading file '%s' (%d) (%d)" % (path, len(s), i))
            if not integer:
                energy = float(s[0])
            f[:, i] = [float(s[1]), float(s[2]), float(s[3])]
            i += 1
            if i == n:
                break
    if i != n:
        raise ValueError("Error while reading file '%s' (%d)" % (path, i))
    return (f, energy) if with_energy else f


def write_exact_forces(path, f, fk):
    """Write_exact_forces (io.c:159-177): 'id F(3) F_k(3)' with %lf."""
    with open(path, "w") as fh:
        for i in range(f.shape[1]):
            fh.write("%d\t%f\t%f\t%f\t%f\t%f\t%f\n" % (i, f[0, i], f[1, i], f[2, i], fk[0, i], fk[1, i], fk[2, i]))


def rms_error(f, ref):
    """DeltaF = sqrt(sum |F - F_ref|^2) / sqrt(N) (error.c:21-34, main.c:446)."""
    f = np.asarray(f)
    return float(np.sqrt(np.sum((f - ref) ** 2)) / np.sqrt(f.shape[-1]))


def alpha_sweep(alphamin, alphamax, alphastep):
    """The reference's alpha loop values (main.c:375): double accumulation."""
    out = []
    a = float(alphamin)
    while a <= alphamax:
        out.append(a)
        a += alphastep
    return out
