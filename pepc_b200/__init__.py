"""pepc_b200 -- Python binding of libpepcg, the B200-native (sm_100a) tree-code
force evaluation that replaces PEPC's pepc_grow_tree / pepc_traverse_tree for
one MPI rank on one GPU.

The binding mirrors the reference's library interface
(src/treecode/lpepcsrc/module_pepc.f90):

    tc = TreeCode(theta2=0.36, eps2=1e-4)       # pepc_initialize + read parameters
    g = tc.pepc_grow_tree(x, y, z, q)            # keys, sort, tree, multipoles
    r = tc.pepc_traverse_tree(g.x, g.y, g.z, keys=g.key)   # fields on targets
    tc.pepc_timber_tree()

Arrays are numpy (host) or torch CUDA tensors (device, through the *_device
methods).  The compute path is the CUDA library only: if libpepcg.so is not
built or no CUDA device is present, the calls raise PepcgError -- there is no
CPU fallback.
"""
import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libpepcg.so")

PEPCG_OK = 0
PEPCG_ERR_BAD_ARG = 1
PEPCG_ERR_CUDA = 2
PEPCG_ERR_OOM = 3
PEPCG_ERR_NODE_POOL = 4
PEPCG_ERR_MAXLEVEL = 5
PEPCG_ERR_INCOMPLETE_WALK = 6
PEPCG_ERR_TIMEOUT = 7
PEPCG_ERR_NO_TREE = 8
PEPCG_ERR_UNSUPPORTED = 9
PEPCG_WARN_NOT_NEUTRAL = 100

CURVE_HILBERT, CURVE_MORTON = 0, 1
PRECISION_PLAIN, PRECISION_MIXED, PRECISION_MIXED_STRICT = 0, 1, 2
WALK_PER_TARGET, WALK_PER_TILE, WALK_GROUP = 0, 1, 2

D = C.POINTER(C.c_double)
I64 = C.POINTER(C.c_int64)
I32 = C.POINTER(C.c_int32)


class PepcgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pepcg error {code}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [
        ("theta2", C.c_double),
        ("eps2", C.c_double),
        ("force_law", C.c_int32),
        ("mac_select", C.c_int32),
        ("curve", C.c_int32),
        ("precision", C.c_int32),
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
        ("device", C.c_int32),
        ("overwrite_results", C.c_int32),
        ("kelbg_invsqrttemp", C.c_double),
        ("group_size", C.c_int32),
        ("reserved0", C.c_int32),
        ("spatial_interaction_cutoff", C.c_double * 3),
        ("reserved", C.c_int32 * 4),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("npart", C.c_int64),
        ("nleaf", C.c_int64),
        ("ntwig", C.c_int64),
        ("max_level", C.c_int64),
        ("dup_count", C.c_int64),
        ("interactions", C.c_int64),
        ("leaf_interactions", C.c_int64),
        ("twig_interactions", C.c_int64),
        ("mac_evaluations", C.c_int64),
        ("t_keys_ms", C.c_double),
        ("t_sort_ms", C.c_double),
        ("t_tree_ms", C.c_double),
        ("t_upward_ms", C.c_double),
        ("t_walk_ms", C.c_double),
        ("t_lattice_ms", C.c_double),
        ("box", C.c_double * 9),
    ]

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if name == "box" else v
        return out


# every symbol declared in include/pepcg.h
EXPORTS = [
    "pepcg_params_default", "pepcg_create", "pepcg_destroy", "pepcg_last_error",
    "pepcg_set_params", "pepcg_grow_tree", "pepcg_grow_tree_device",
    "pepcg_get_particles_device", "pepcg_traverse_tree", "pepcg_traverse_tree_device",
    "pepcg_traverse_self_device", "pepcg_timber_tree", "pepcg_stats_get", "pepcg_num_nodes",
    "pepcg_tree_export", "pepcg_direct", "pepcg_lattice", "pepcg_multipole_from_particle",
    "pepcg_shift_multipoles_up", "pepcg_force_with_leaf", "pepcg_force_with_twig", "pepcg_mac",
    "pepcg_set_stream", "pepcg_kernel_launches", "pepcg_sort_keys_noalloc",
    "pepcg_traverse_adjoint", "pepcg_traverse_adjoint_device",
    "pepcg_push_particles_device", "pepcg_apply_external_field_device",
    "pepcg_potential_energy_device",
    "pepcg_constrain_periodic_device", "pepcg_gather_device",
    "pepcg_traverse_range_device", "pepcg_restore_device",
    "pepcg_sort_keys", "pepcg_sort_keys_device", "pepcg_lattice_force",
    "pepcg_debug_fail_allocations",
]

_LIB = None


def lib():
    """Load libpepcg.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIBPATH):
        raise PepcgError(-1, f"{LIBPATH} is not built; run python -m pepc_b200.build")
    L = C.CDLL(LIBPATH)
    VP = C.c_void_p
    L.pepcg_params_default.argtypes = [C.POINTER(Params)]
    L.pepcg_params_default.restype = None
    L.pepcg_create.argtypes = [C.POINTER(VP), C.POINTER(Params)]
    L.pepcg_destroy.argtypes = [VP]
    L.pepcg_last_error.argtypes = [VP]
    L.pepcg_last_error.restype = C.c_char_p
    L.pepcg_set_params.argtypes = [VP, C.POINTER(Params)]
    L.pepcg_grow_tree.argtypes = [VP, C.c_int64, D, D, D, D, I64, I64, D, D, D]
    L.pepcg_grow_tree_device.argtypes = [VP, C.c_int64, VP, VP, VP, VP]
    L.pepcg_get_particles_device.argtypes = [VP, VP, VP, VP, VP, VP, VP]
    L.pepcg_traverse_tree.argtypes = [VP, C.c_int64, D, D, D, I64, D, D, D, D, D]
    L.pepcg_traverse_tree_device.argtypes = [VP, C.c_int64, VP, VP, VP, VP, VP, VP, VP, VP, VP]
    L.pepcg_traverse_self_device.argtypes = [VP, VP, VP, VP, VP, VP]
    L.pepcg_timber_tree.argtypes = [VP]
    L.pepcg_set_stream.argtypes = [VP, VP]
    L.pepcg_sort_keys_noalloc.argtypes = [C.c_int64, VP, VP, VP, VP]
    L.pepcg_sort_keys.argtypes = [VP, C.c_int64, I64, I64, I64]
    L.pepcg_sort_keys_device.argtypes = [VP, C.c_int64, VP, VP, VP]
    L.pepcg_traverse_adjoint.argtypes = [VP, C.c_int64, D, D, D, D, D, D, D, D, D, D, D]
    L.pepcg_traverse_adjoint_device.argtypes = [VP, C.c_int64] + [VP] * 11
    L.pepcg_push_particles_device.argtypes = [VP, C.c_int64, C.c_double] + [VP] * 11
    L.pepcg_apply_external_field_device.argtypes = [VP, C.c_int64, C.c_double, VP, VP, VP]
    L.pepcg_potential_energy_device.argtypes = [VP, C.c_int64, VP, VP, C.POINTER(C.c_double)]
    L.pepcg_constrain_periodic_device.argtypes = [VP, C.c_int64, VP, VP, VP]
    L.pepcg_gather_device.argtypes = [VP, VP, VP]
    L.pepcg_traverse_range_device.argtypes = [VP, C.c_int64, C.c_int64, VP, VP, VP, VP, VP]
    L.pepcg_restore_device.argtypes = [VP, VP, VP]
    L.pepcg_debug_fail_allocations.argtypes = [C.c_int64]
    L.pepcg_debug_fail_allocations.restype = None
    L.pepcg_kernel_launches.argtypes = []
    L.pepcg_kernel_launches.restype = C.c_longlong
    L.pepcg_stats_get.argtypes = [VP, C.POINTER(Stats)]
    L.pepcg_num_nodes.argtypes = [VP]
    L.pepcg_num_nodes.restype = C.c_int64
    L.pepcg_tree_export.argtypes = [VP, I64, I32, I64, I64, I64, I64, I64, D]
    L.pepcg_direct.argtypes = [VP, C.c_int64, I64, D, D, D, D]
    L.pepcg_lattice.argtypes = [VP, C.c_int64, D, D, D, D, D, D, D]
    L.pepcg_lattice_force.argtypes = [VP, D, D, D]
    L.pepcg_multipole_from_particle.argtypes = [D, C.c_double, D]
    L.pepcg_shift_multipoles_up.argtypes = [D, D, C.c_int32]
    L.pepcg_force_with_leaf.argtypes = [D, D, C.c_double, C.c_double, D, D]
    L.pepcg_force_with_twig.argtypes = [D, D, C.c_double, C.c_double, D, D]
    L.pepcg_mac.argtypes = [C.c_double, C.c_double, C.c_double, I32]
    _LIB = L
    return L


def _dp(a):
    return a.ctypes.data_as(D)


def _ip(a):
    return a.ctypes.data_as(I64)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _tptr(t):
    """Device pointer of a contiguous torch CUDA tensor."""
    if not (hasattr(t, "is_cuda") and t.is_cuda and t.is_contiguous()):
        raise PepcgError(PEPCG_ERR_BAD_ARG, "expected a contiguous CUDA tensor")
    return C.c_void_p(t.data_ptr())


def make_params(**kw):
    p = Params()
    lib().pepcg_params_default(C.byref(p))
    for k, v in kw.items():
        if k in ("periodicity", "t_lattice_1", "t_lattice_2", "t_lattice_3", "lattice_origin",
                 "spatial_interaction_cutoff"):
            arr = getattr(p, k)
            for i in range(3):
                arr[i] = v[i]
        else:
            if not hasattr(p, k):
                raise PepcgError(PEPCG_ERR_BAD_ARG, f"unknown parameter {k}")
            setattr(p, k, v)
    return p


@dataclass
class Grown:
    key: np.ndarray
    perm: np.ndarray
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray


class TreeCode:
    """One context of libpepcg (one GPU, one rank)."""

    def __init__(self, **params):
        self._h = C.c_void_p()
        self.last_status = PEPCG_OK
        self.params = make_params(**params)
        rc = lib().pepcg_create(C.byref(self._h), C.byref(self.params))
        if rc != PEPCG_OK:
            raise PepcgError(rc, lib().pepcg_last_error(None).decode())

    # -- helpers
    def _check(self, rc, allow_warn=True):
        self.last_status = rc
        if rc == PEPCG_OK or (allow_warn and rc == PEPCG_WARN_NOT_NEUTRAL):
            return rc
        raise PepcgError(rc, lib().pepcg_last_error(self._h).decode())

    def close(self):
        if self._h:
            lib().pepcg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, **kw):
        for k, v in kw.items():
            if k in ("spatial_interaction_cutoff",):
                arr = getattr(self.params, k)
                for i in range(3):
                    arr[i] = v[i]
            else:
                setattr(self.params, k, v)
        self._check(lib().pepcg_set_params(self._h, C.byref(self.params)))

    # -- the reference's entry points (module_pepc.f90)
    def pepc_grow_tree(self, x, y, z, q):
        n = len(x)
        x, y, z, q = _f64(x), _f64(y), _f64(z), _f64(q)
        key = np.zeros(n, np.int64)
        perm = np.zeros(n, np.int64)
        xo, yo, zo = np.zeros(n), np.zeros(n), np.zeros(n)
        self._check(lib().pepcg_grow_tree(self._h, n, _dp(x), _dp(y), _dp(z), _dp(q), _ip(key),
                                          _ip(perm), _dp(xo), _dp(yo), _dp(zo)))
        return Grown(key, perm, xo, yo, zo)

    def pepc_traverse_tree(self, x, y, z, keys=None, e=None, pot=None, work=None):
        """Fields on targets; accumulates onto e/pot/work when given (like particle%results)."""
        n = len(x)
        x, y, z = _f64(x), _f64(y), _f64(z)
        ex = np.zeros(n) if e is None else _f64(e[0]).copy()
        ey = np.zeros(n) if e is None else _f64(e[1]).copy()
        ez = np.zeros(n) if e is None else _f64(e[2]).copy()
        pt = np.zeros(n) if pot is None else _f64(pot).copy()
        wk = np.zeros(n) if work is None else _f64(work).copy()
        kp = None
        if keys is not None:
            keys = np.ascontiguousarray(keys, dtype=np.int64)
            kp = _ip(keys)
        self._check(lib().pepcg_traverse_tree(self._h, n, _dp(x), _dp(y), _dp(z), kp, _dp(ex),
                                              _dp(ey), _dp(ez), _dp(pt), _dp(wk)))
        return dict(ex=ex, ey=ey, ez=ez, pot=pt, work=wk)

    def sort_keys(self, keys):
        """The local key sort of domain_decompose (slsort_keys at one rank):
        sorted keys and the 0-based input index of each, with equal keys in
        the reference's order."""
        keys = np.ascontiguousarray(keys, dtype=np.int64)
        n = len(keys)
        ko = np.zeros(n, np.int64)
        po = np.zeros(n, np.int64)
        self._check(lib().pepcg_sort_keys(self._h, n, _ip(keys), _ip(ko), _ip(po)))
        return ko, po

    def sort_keys_device(self, keys, keys_out, perm_out):
        return self._check(lib().pepcg_sort_keys_device(self._h, keys.numel(), _tptr(keys),
                                                        _tptr(keys_out), _tptr(perm_out)))

    def pepc_timber_tree(self):
        self._check(lib().pepcg_timber_tree(self._h))

    # -- device-resident variants (torch CUDA float64 tensors)
    def grow_tree_device(self, x, y, z, q):
        return self._check(lib().pepcg_grow_tree_device(self._h, x.numel(), _tptr(x), _tptr(y),
                                                        _tptr(z), _tptr(q)))

    def traverse_self_device(self, ex, ey, ez, pot, work):
        return self._check(lib().pepcg_traverse_self_device(self._h, _tptr(ex), _tptr(ey),
                                                            _tptr(ez), _tptr(pot), _tptr(work)))

    def traverse_tree_device(self, x, y, z, ex, ey, ez, pot, work, keys=None):
        kp = _tptr(keys) if keys is not None else None
        return self._check(lib().pepcg_traverse_tree_device(
            self._h, x.numel(), _tptr(x), _tptr(y), _tptr(z), kp, _tptr(ex), _tptr(ey),
            _tptr(ez), _tptr(pot), _tptr(work)))

    def particles_device(self, key, perm, x, y, z, q):
        return self._check(lib().pepcg_get_particles_device(
            self._h, _tptr(key), _tptr(perm), _tptr(x), _tptr(y), _tptr(z), _tptr(q)))

    # -- the frontend's time step on device arrays (module_helper.f90:205-222, :321-334;
    #    module_mirror_boxes.f90:177-218)
    def push_particles_device(self, dt, q, m, e, v, x):
        """v += dt q/m E, then x += dt v; e, v, x are (x, y, z) triples of tensors."""
        ptrs = [_tptr(t) for t in (q, m, *e, *v, *x)]
        return self._check(lib().pepcg_push_particles_device(self._h, q.numel(), float(dt), *ptrs))

    def apply_external_field_device(self, ez_ext, z, ez, pot):
        return self._check(lib().pepcg_apply_external_field_device(
            self._h, z.numel(), float(ez_ext), _tptr(z), _tptr(ez), _tptr(pot)))

    def potential_energy_device(self, q, pot):
        """sum of 0.5 q phi over device arrays, in FP64 on the device (pepc-b's
        potenergy, module_diagnostics.f90:227-263)."""
        e = C.c_double(0.0)
        self._check(lib().pepcg_potential_energy_device(self._h, q.numel(), _tptr(q), _tptr(pot),
                                                        C.byref(e)))
        return e.value

    def constrain_periodic_device(self, x, y, z):
        return self._check(lib().pepcg_constrain_periodic_device(self._h, x.numel(), _tptr(x),
                                                                 _tptr(y), _tptr(z)))

    def gather_device(self, src, dst):
        """dst[i] = src[perm[i]] with the last grow's permutation (key order)."""
        return self._check(lib().pepcg_gather_device(self._h, _tptr(src), _tptr(dst)))

    def traverse_range_device(self, t0, t1, ex, ey, ez, pot, work):
        """Fields on the grown particles [t0, t1) of the key order (one rank's share)."""
        return self._check(lib().pepcg_traverse_range_device(
            self._h, int(t0), int(t1), _tptr(ex), _tptr(ey), _tptr(ez), _tptr(pot), _tptr(work)))

    def restore_device(self, src, dst):
        """dst[perm[i]] = src[i]: a key-ordered array back to the last grow's input order."""
        return self._check(lib().pepcg_restore_device(self._h, _tptr(src), _tptr(dst)))

    def set_stream(self, stream_ptr):
        """Launch on an external cudaStream_t (int handle, e.g. torch's
        ``Stream.cuda_stream``); 0 is the legacy default stream (passed on as
        cudaStreamLegacy, since NULL asks the library for a private stream);
        None selects a private stream."""
        if stream_ptr is None:
            h = None
        elif stream_ptr == 0:
            h = C.c_void_p(1)  # cudaStreamLegacy
        else:
            h = C.c_void_p(stream_ptr)
        self._check(lib().pepcg_set_stream(self._h, h))

    # -- diagnostics
    def stats(self):
        s = Stats()
        self._check(lib().pepcg_stats_get(self._h, C.byref(s)))
        return s.as_dict()

    def tree(self):
        n = lib().pepcg_num_nodes(self._h)
        out = dict(key=np.zeros(n, np.int64), level=np.zeros(n, np.int32),
                   leaves=np.zeros(n, np.int64), descendants=np.zeros(n, np.int64),
                   parent=np.zeros(n, np.int64), first_child=np.zeros(n, np.int64),
                   next_sibling=np.zeros(n, np.int64), moments=np.zeros((n, 15)))
        self._check(lib().pepcg_tree_export(
            self._h, _ip(out["key"]), out["level"].ctypes.data_as(I32), _ip(out["leaves"]),
            _ip(out["descendants"]), _ip(out["parent"]), _ip(out["first_child"]),
            _ip(out["next_sibling"]), _dp(out["moments"])))
        return out

    def direct(self, tidx):
        tidx = np.ascontiguousarray(tidx, dtype=np.int64)
        n = len(tidx)
        ex, ey, ez, pt = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
        self._check(lib().pepcg_direct(self._h, n, _ip(tidx), _dp(ex), _dp(ey), _dp(ez), _dp(pt)))
        return dict(ex=ex, ey=ey, ez=ez, pot=pt)

    def traverse_adjoint(self, x, y, z, dLdE, dLdphi, npart):
        """dL/dq, dL/dx of the grown particles (caller's original order) for
        dL/dE = (3 arrays) and dL/dphi at the targets x, y, z."""
        nt = len(x)
        args = [_f64(v) for v in (x, y, z, dLdE[0], dLdE[1], dLdE[2], dLdphi)]
        out = [np.zeros(npart) for _ in range(4)]
        self._check(lib().pepcg_traverse_adjoint(self._h, nt, *[_dp(a) for a in args],
                                                 *[_dp(o) for o in out]))
        return dict(q=out[0], x=out[1], y=out[2], z=out[3])

    def traverse_adjoint_device(self, x, y, z, dLdE, dLdphi, dq, dx, dy, dz):
        """traverse_adjoint on torch CUDA float64 tensors; dq..dz are overwritten."""
        ptrs = [_tptr(t) for t in (x, y, z, dLdE[0], dLdE[1], dLdE[2], dLdphi, dq, dx, dy, dz)]
        return self._check(lib().pepcg_traverse_adjoint_device(self._h, x.numel(), *ptrs))

    def lattice_force(self, pos):
        """fmm_sum_lattice_force at one position: (e[3], phi)."""
        e = np.zeros(3)
        phi = np.zeros(1)
        self._check(lib().pepcg_lattice_force(self._h, _dp(_f64(pos)), _dp(e), _dp(phi)))
        return e, phi[0]

    def lattice(self, x, y, z):
        n = len(x)
        x, y, z = _f64(x), _f64(y), _f64(z)
        ex, ey, ez, pt = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
        self._check(lib().pepcg_lattice(self._h, n, _dp(x), _dp(y), _dp(z), _dp(ex), _dp(ey),
                                         _dp(ez), _dp(pt)))
        return dict(ex=ex, ey=ey, ez=ez, pot=pt)


# -- scalar backend API (coulomb/module_interaction_specific.f90:46-60)
def _chk(rc):
    if rc != PEPCG_OK:
        raise PepcgError(rc, lib().pepcg_last_error(None).decode())


def multipole_from_particle(pos, q):
    out = np.zeros(15)
    _chk(lib().pepcg_multipole_from_particle(_dp(_f64(pos)), float(q), _dp(out)))
    return out


def shift_multipoles_up(children):
    ch = _f64(np.asarray(children).reshape(-1, 15))
    out = np.zeros(15)
    _chk(lib().pepcg_shift_multipoles_up(_dp(out), _dp(ch), ch.shape[0]))
    return out


def force_with_leaf(node, delta, dist2, eps2):
    e = np.zeros(3)
    phi = np.zeros(1)
    _chk(lib().pepcg_force_with_leaf(_dp(_f64(node)), _dp(_f64(delta)), float(dist2), float(eps2),
                                     _dp(e), _dp(phi)))
    return e, phi[0]


def force_with_twig(node, delta, dist2, eps2):
    e = np.zeros(3)
    phi = np.zeros(1)
    _chk(lib().pepcg_force_with_twig(_dp(_f64(node)), _dp(_f64(delta)), float(dist2), float(eps2),
                                     _dp(e), _dp(phi)))
    return e, phi[0]


def kernel_launches():
    return int(lib().pepcg_kernel_launches())


def mac(theta2, dist2, boxlength2):
    a = C.c_int32(0)
    _chk(lib().pepcg_mac(float(theta2), float(dist2), float(boxlength2), C.byref(a)))
    return bool(a.value)


def shard_range(n, rank, world, align=64):
    """[t0, t1) of the key-ordered targets for one of `world` ranks: contiguous,
    disjoint, covering [0, n), with every boundary a multiple of `align` so each
    rank's group-walk buckets (32 or 64 targets) are the single-GPU ones."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    blocks = (n + align - 1) // align
    b0 = blocks * rank // world
    b1 = blocks * (rank + 1) // world
    return min(n, b0 * align), min(n, b1 * align)


def gather_shards(local, n, rank, world, align=64, group=None):
    """The exchange of a target-sharded traverse: every rank's share of the
    key-ordered fields (local: a (k, t1 - t0) tensor of this rank's
    shard_range share, k fields) gathered on every rank as a (k, n) tensor.
    The shares are padded to the largest one so that a single all-gather
    moves them (all_gather_into_tensor over NCCL; a list all-gather where the
    backend has no tensor form)."""
    import torch
    import torch.distributed as dist
    sizes = [shard_range(n, r, world, align) for r in range(world)]
    t0, t1 = sizes[rank]
    if local.dim() != 2 or local.shape[1] != t1 - t0:
        raise ValueError(f"rank {rank}: local share must be (k, {t1 - t0}), got {tuple(local.shape)}")
    k = local.shape[0]
    cap = max(b - a for a, b in sizes)
    buf = torch.zeros((k, cap), dtype=local.dtype, device=local.device)
    buf[:, : t1 - t0] = local
    if world == 1:
        return buf[:, :n].clone()
    try:
        flat = torch.empty((world, k, cap), dtype=local.dtype, device=local.device)
        dist.all_gather_into_tensor(flat, buf, group=group)
        parts = [flat[r] for r in range(world)]
    except (RuntimeError, NotImplementedError):
        parts = [torch.empty_like(buf) for _ in range(world)]
        dist.all_gather(parts, buf, group=group)
    return torch.cat([parts[r][:, : b - a] for r, (a, b) in enumerate(sizes)], dim=1)

