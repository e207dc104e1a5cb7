"""ctypes access to the CPU parity checker (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py.  The product (pepc_b200) never imports this.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None

D = C.POINTER(C.c_double)
I64 = C.POINTER(C.c_int64)
I32 = C.POINTER(C.c_int32)


class OrcParams(C.Structure):
    _fields_ = [
        ("theta2", C.c_double),
        ("eps2", C.c_double),
        ("curve", C.c_int32),
        ("walk", C.c_int32),
        ("tile_size", C.c_int32),
        ("force_cubic_domain", C.c_int32),
        ("periodicity", C.c_int32 * 3),
        ("mirror_box_layers", C.c_int32),
        ("include_far_field_if_periodic", C.c_int32),
        ("fmm_extrinsic_correction", C.c_int32),
        ("t_lattice_1", C.c_double * 3),
        ("t_lattice_2", C.c_double * 3),
        ("t_lattice_3", C.c_double * 3),
        ("lattice_origin", C.c_double * 3),
        ("num_threads", C.c_int32),
        ("mac_select", C.c_int32),
        ("force_law", C.c_int32),
        ("kelbg_invsqrttemp", C.c_double),
        ("spatial_interaction_cutoff", C.c_double * 3),
    ]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle/liboracle.so is not built (run make -C oracle)")
        L = C.CDLL(path)
        L.orc_params_default.argtypes = [C.POINTER(OrcParams)]
        L.orc_box_create.argtypes = [C.c_int64, D, D, D, C.c_int32, D]
        L.orc_compute_keys.argtypes = [C.c_int64, D, D, D, D, D, C.c_int32, I64]
        L.orc_key_to_coord.argtypes = [C.c_int64, D, D, C.c_int32, D]
        L.orc_sort_radix.argtypes = [C.c_int64, I64, I64]
        L.orc_multipole_from_particle.argtypes = [D, C.c_double, D]
        L.orc_shift_multipoles_up.argtypes = [D, D, C.c_int32]
        L.orc_force_leaf.argtypes = [D, D, C.c_double, D, D]
        L.orc_force_twig.argtypes = [D, D, C.c_double, D, D]
        L.orc_par_rand.argtypes = [C.c_int32, C.c_int64, D]
        L.orc_create.argtypes = [C.POINTER(OrcParams)]
        L.orc_create.restype = C.c_void_p
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_grow_tree.argtypes = [C.c_void_p, C.c_int64, D, D, D, D, I64, I64, D, D, D, D]
        L.orc_grow_tree.restype = C.c_int
        L.orc_traverse_tree.argtypes = [C.c_void_p, C.c_int64, D, D, D, I64, D, D, D, D, D]
        L.orc_traverse_tree.restype = C.c_int
        L.orc_num_nodes.argtypes = [C.c_void_p]
        L.orc_num_nodes.restype = C.c_int64
        L.orc_tree_export.argtypes = [C.c_void_p, I64, I32, I64, I64, I64, I64, I64, D]
        L.orc_box.argtypes = [C.c_void_p, D]
        L.orc_counters.argtypes = [C.c_void_p, I64]
        L.orc_direct.argtypes = [C.c_void_p, C.c_int64, I64, D, D, D, D]
        L.orc_direct.restype = C.c_int
        L.orc_lattice.argtypes = [C.c_void_p, C.c_int64, D, D, D, D, D, D, D]
        L.orc_lattice.restype = C.c_int
        L.orc_fmm_lattice_coefficients.argtypes = [C.POINTER(OrcParams), D]
        L.orc_set_lattice_coefficients.argtypes = [C.c_void_p, D]
        L.orc_traverse_adjoint.argtypes = [C.c_void_p, C.c_int64, D, D, D, D, D, D, D, D, D, D, D]
        L.orc_traverse_adjoint.restype = C.c_int
        L.orc_direct_adjoint.argtypes = [C.c_void_p, C.c_int64, D, D, D, D, D, D, D, D, D, D, D]
        L.orc_direct_adjoint.restype = C.c_int
        L.orc_set_lattice_coefficients.restype = C.c_int
        L.orc_push_particles.argtypes = [C.c_int64, C.c_double] + [D] * 11
        L.orc_apply_external_field.argtypes = [C.c_int64, C.c_double, D, D, D]
        L.orc_constrain_periodic.argtypes = [C.POINTER(OrcParams), C.c_int64, D, D, D]
        _LIB = L
    return _LIB


def ref_lib():
    """The reference's own sort, compiled from its sources into oracle/_ref."""
    global _REF
    if _REF is None:
        path = os.path.join(HERE, "_ref", "libslref.so")
        if not os.path.exists(path):
            return None
        R = C.CDLL(path)
        R.ref_sort_keys.argtypes = [C.c_int64, I64, I64]
        R.ref_sort_keys.restype = C.c_int
        _REF = R
    return _REF


def dp(a):
    return a.ctypes.data_as(D)


def ip(a):
    return a.ctypes.data_as(I64)


def i32p(a):
    return a.ctypes.data_as(I32)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def params(**kw):
    p = OrcParams()
    lib().orc_params_default(C.byref(p))
    for k, v in kw.items():
        if k in ("periodicity", "t_lattice_1", "t_lattice_2", "t_lattice_3", "lattice_origin",
                 "spatial_interaction_cutoff"):
            arr = getattr(p, k)
            for i in range(3):
                arr[i] = v[i]
        else:
            setattr(p, k, v)
    return p


def box_create(x, y, z, force_cubic=False):
    x, y, z = f64(x), f64(y), f64(z)
    out = np.zeros(9)
    lib().orc_box_create(len(x), dp(x), dp(y), dp(z), int(force_cubic), dp(out))
    return out


def compute_keys(x, y, z, boxmin, boxsize, curve=0):
    x, y, z = f64(x), f64(y), f64(z)
    bm, bs = f64(boxmin), f64(boxsize)
    k = np.zeros(len(x), dtype=np.int64)
    lib().orc_compute_keys(len(x), dp(x), dp(y), dp(z), dp(bm), dp(bs), curve, ip(k))
    return k


def key_to_coord(key, boxmin, boxsize, curve=0):
    bm, bs = f64(boxmin), f64(boxsize)
    out = np.zeros(3)
    lib().orc_key_to_coord(int(key), dp(bm), dp(bs), curve, dp(out))
    return out


def sort_radix(keys):
    k = np.array(keys, dtype=np.int64)
    idx = np.arange(len(k), dtype=np.int64)
    lib().orc_sort_radix(len(k), ip(k), ip(idx))
    return k, idx


def ref_sort(keys):
    R = ref_lib()
    if R is None:
        return None
    k = np.array(keys, dtype=np.int64)
    idx = np.zeros(len(k), dtype=np.int64)
    R.ref_sort_keys(len(k), ip(k), ip(idx))
    return k, idx


def par_rand(iseed, n):
    out = np.zeros(n)
    lib().orc_par_rand(int(iseed), int(n), dp(out))
    return out


GOLDEN = os.path.join(HERE, "..", "tests", "golden", "reference_pins.npz")


def unit_cube(p):
    """system_is_unit_cube (module_mirror_boxes.f90:248-255)."""
    a, b, c = p.t_lattice_1, p.t_lattice_2, p.t_lattice_3
    axes = (a[0] > 0 and a[1] == 0 and a[2] == 0 and b[0] == 0 and b[1] > 0 and b[2] == 0
            and c[0] == 0 and c[1] == 0 and c[2] > 0)
    nsq = lambda v: (v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]  # noqa: E731
    return axes and nsq(a) == 1.0 and nsq(b) == 1.0 and nsq(c) == 1.0


def reference_lattice_table(gold):
    """The reference's pretabulated unit-cube MLattice (l <= 40) from the golden fixture."""
    ml = np.zeros(861, dtype=np.complex128)
    for l, m, v in zip(gold["lattice_l"], gold["lattice_m"], gold["lattice_v"]):
        if l <= 40:
            ml[l * (l + 1) // 2 + m] = v
    return ml


def lattice_coefficients(p):
    out = np.zeros(2 * 861)
    lib().orc_fmm_lattice_coefficients(C.byref(p), dp(out))
    return out[0::2] + 1j * out[1::2]


class Oracle:
    """Whole-path CPU restatement with the same call shape as pepc_b200.TreeCode."""

    def __init__(self, **kw):
        self.p = params(**kw)
        self.h = lib().orc_create(C.byref(self.p))
        # fmm_framework_prepare (module_fmm_framework.f90:112-115): a unit-cube
        # lattice loads the pretabulated coefficients instead of iterating
        if (any(self.p.periodicity) and self.p.include_far_field_if_periodic
                and unit_cube(self.p)):
            self.set_lattice_coefficients(reference_lattice_table(np.load(GOLDEN)))

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def grow_tree(self, x, y, z, q):
        n = len(x)
        x, y, z, q = f64(x), f64(y), f64(z), f64(q)
        key = np.zeros(n, dtype=np.int64)
        perm = np.zeros(n, dtype=np.int64)
        xo, yo, zo, qo = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
        rc = lib().orc_grow_tree(self.h, n, dp(x), dp(y), dp(z), dp(q), ip(key), ip(perm),
                                 dp(xo), dp(yo), dp(zo), dp(qo))
        if rc != 0:
            raise RuntimeError(f"orc_grow_tree failed: {rc}")
        return dict(key=key, perm=perm, x=xo, y=yo, z=zo, q=qo)

    def traverse_tree(self, x, y, z, keys=None, e=None, pot=None, work=None):
        n = len(x)
        x, y, z = f64(x), f64(y), f64(z)
        ex = np.zeros(n) if e is None else f64(e[0]).copy()
        ey = np.zeros(n) if e is None else f64(e[1]).copy()
        ez = np.zeros(n) if e is None else f64(e[2]).copy()
        pt = np.zeros(n) if pot is None else f64(pot).copy()
        wk = np.zeros(n) if work is None else f64(work).copy()
        kp = None
        if keys is not None:
            keys = np.ascontiguousarray(keys, dtype=np.int64)
            kp = ip(keys)
        rc = lib().orc_traverse_tree(self.h, n, dp(x), dp(y), dp(z), kp, dp(ex), dp(ey), dp(ez),
                                     dp(pt), dp(wk))
        if rc != 0:
            raise RuntimeError(f"orc_traverse_tree failed: {rc}")
        return dict(ex=ex, ey=ey, ez=ez, pot=pt, work=wk)

    def tree(self):
        n = lib().orc_num_nodes(self.h)
        out = dict(key=np.zeros(n, np.int64), level=np.zeros(n, np.int32),
                   leaves=np.zeros(n, np.int64), descendants=np.zeros(n, np.int64),
                   parent=np.zeros(n, np.int64), first_child=np.zeros(n, np.int64),
                   next_sibling=np.zeros(n, np.int64), moments=np.zeros((n, 15)))
        lib().orc_tree_export(self.h, ip(out["key"]), i32p(out["level"]), ip(out["leaves"]),
                              ip(out["descendants"]), ip(out["parent"]), ip(out["first_child"]),
                              ip(out["next_sibling"]), dp(out["moments"]))
        return out

    def box(self):
        out = np.zeros(9)
        lib().orc_box(self.h, dp(out))
        return out

    def counters(self):
        out = np.zeros(2, np.int64)
        lib().orc_counters(self.h, ip(out))
        return dict(interactions=int(out[0]), mac_evaluations=int(out[1]))

    def direct(self, tidx):
        tidx = np.ascontiguousarray(tidx, dtype=np.int64)
        n = len(tidx)
        ex, ey, ez, pt = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
        rc = lib().orc_direct(self.h, n, ip(tidx), dp(ex), dp(ey), dp(ez), dp(pt))
        if rc != 0:
            raise RuntimeError(f"orc_direct failed: {rc}")
        return dict(ex=ex, ey=ey, ez=ez, pot=pt)

    def traverse_adjoint(self, x, y, z, gE, gphi, npart, direct=False):
        """dL/dq, dL/dx (original particle order) of sum_t gphi phi_t + gE.E_t."""
        nt = len(x)
        args = [f64(v) for v in (x, y, z, gE[0], gE[1], gE[2], gphi)]
        out = [np.zeros(npart) for _ in range(4)]
        fn = lib().orc_direct_adjoint if direct else lib().orc_traverse_adjoint
        rc = fn(self.h, nt, *[dp(a) for a in args], *[dp(o) for o in out])
        if rc != 0:
            raise RuntimeError(f"adjoint failed: {rc}")
        return dict(q=out[0], x=out[1], y=out[2], z=out[3])

    def set_lattice_coefficients(self, ml):
        ml = np.asarray(ml, dtype=np.complex128)
        buf = np.ascontiguousarray(np.stack([ml.real, ml.imag], axis=1).reshape(-1))
        if lib().orc_set_lattice_coefficients(self.h, dp(buf)) != 0:
            raise RuntimeError("not a periodic context")

    def lattice(self, x, y, z):
        n = len(x)
        x, y, z = f64(x), f64(y), f64(z)
        ex, ey, ez, pt = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
        rc = lib().orc_lattice(self.h, n, dp(x), dp(y), dp(z), dp(ex), dp(ey), dp(ez), dp(pt))
        if rc != 0:
            raise RuntimeError("lattice term needs a periodic context")
        return dict(ex=ex, ey=ey, ez=ez, pot=pt)


def push_particles(dt, q, m, e, v, x):
    """pepc-mini push_particles on numpy arrays (v, x updated in place)."""
    args = [f64(a) for a in (q, m, *e)]
    for a in (*v, *x):
        assert a.dtype == np.float64 and a.flags.c_contiguous
    lib().orc_push_particles(len(q), dt, *[dp(a) for a in args],
                             *[dp(a) for a in (*v, *x)])


def apply_external_field(ez_ext, z, ez, pot):
    lib().orc_apply_external_field(len(z), ez_ext, dp(f64(z)), dp(ez), dp(pot))


def constrain_periodic(x, y, z, **kw):
    """constrain_periodic with the lattice of params(**kw); x, y, z in place."""
    p = params(**kw)
    lib().orc_constrain_periodic(C.byref(p), len(x), dp(x), dp(y), dp(z))

