"""ctypes front end of librsd_cuda.so, the sm_100a C-ABI backend for the Residuum heat-equation
hot path (declared in include/rsd.h).

This is the binding a Python caller (tests, bench.py, a PyTorch autograd wrapper) uses; C++ callers
use the backend tag in include/rsd_residuum.hpp.  There is no CPU fallback: every call goes to the CUDA
library, and importing raises if the library is missing.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librsd_cuda.so")

_P, _D, _I32, _I64, _SZ = C.c_void_p, C.c_double, C.c_int32, C.c_int64, C.c_size_t

RSD_H2H, RSD_H2D, RSD_D2H, RSD_D2D = 0, 1, 2, 3
CG, GMRES = 0, 1
IDENTITY, JACOBI = 0, 1
FP64, MIXED = 0, 1
RELATIVE, ABSOLUTE = 0, 1
OP_CSR, OP_FEM = 0, 1      # LinearSolverConfig::OperatorType

ERRORS = {-1: "RSD_EINVAL", -2: "RSD_ENOMEM", -3: "RSD_ECUDA", -5: "RSD_EBREAKDOWN", -6: "RSD_ENAN",
          -7: "RSD_EPARSE", -8: "RSD_ETIMEOUT"}


class RsdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Report(C.Structure):
    """rsd_report: SolverReport plus the FP64-checked residual of mixed precision."""
    _fields_ = [("converged", _I32), ("status", _I32), ("iterations", _I64), ("initialResidual", _D),
                ("finalResidual", _D), ("finalResidualRel", _D), ("trueResidualRel", _D), ("refinements", _I64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class SolverConfig(C.Structure):
    _fields_ = [("type", _I32), ("precond", _I32), ("precision", _I32), ("tol_type", _I32), ("tol", _D),
                ("max_iters", _I64), ("krylov_dim", _I64), ("reliable_delta", _D), ("operator_type", _I32),
                ("reserved", _I32)]

    @classmethod
    def make(cls, type=CG, precond=JACOBI, precision=FP64, tol=1e-10, max_iters=1000, krylov_dim=30,
             tol_type=RELATIVE, reliable_delta=0.0, operator_type=OP_CSR):
        return cls(type, precond, precision, tol_type, tol, max_iters, krylov_dim, reliable_delta, operator_type, 0)


class HeatDesc(C.Structure):
    _fields_ = [("nq", _I32), ("k_const", _D), ("k_expr", C.c_char_p), ("dk_expr", C.c_char_p), ("k_elem", _P),
                ("rho", _D), ("cp", _D), ("src_expr", C.c_char_p), ("dirichlet_expr", C.c_char_p * 6),
                ("k_tensor", _P), ("cp_expr", C.c_char_p), ("dcp_expr", C.c_char_p), ("num_dirichlet", _I32),
                ("dirichlet_tags", _P), ("dirichlet_exprs", _P)]


class PmshInfo(C.Structure):
    _fields_ = [("parametric_dim", _I32), ("spatial_dim", _I32), ("family", _I32), ("basis", _I32), ("num_nodes", _I64),
                ("num_elements", _I64), ("nodes_per_element", _I32), ("faces_per_element", _I32), ("num_orders", _I32),
                ("order", _I32 * 3), ("iga", _I32)]


_lib = None

# (name, argtypes) for every entry point of include/rsd.h
SIGNATURES = {
    "rsd_ctx_create": [C.c_int, C.POINTER(_P)],
    "rsd_ctx_destroy": [_P],
    "rsd_ctx_sync": [_P],
    "rsd_ctx_stream": [_P],
    "rsd_last_error_string": [],
    "rsd_version": [C.POINTER(_I32), C.POINTER(_I32)],
    "rsd_expr_check": [C.c_char_p, C.POINTER(_I32)],
    "rsd_ctx_profile": [_P, _I32],
    "rsd_ctx_profile_get": [_P, C.c_char_p, C.POINTER(_I64), C.POINTER(_D)],
    "rsd_alloc": [_P, _SZ, C.POINTER(_P)],
    "rsd_free": [_P, _P],
    "rsd_alloc_managed": [_P, _SZ, C.POINTER(_P)],
    "rsd_memcpy": [_P, _P, _P, _SZ, _I32],
    "rsd_memset_zero": [_P, _P, _SZ],
    "rsd_fill_f64": [_P, _P, _I64, _D],
    "rsd_fill_f32": [_P, _P, _I64, C.c_float],
    "rsd_dot": [_P, _I64, _P, _P, C.POINTER(_D)],
    "rsd_nrm2": [_P, _I64, _P, C.POINTER(_D)],
    "rsd_axpy": [_P, _I64, _D, _P, _P],
    "rsd_axpby": [_P, _I64, _D, _D, _P, _P],
    "rsd_scal": [_P, _I64, _D, _P],
    "rsd_copy": [_P, _I64, _P, _P],
    "rsd_mul": [_P, _I64, _P, _P, _P],
    "rsd_csr_create": [_P, _I64, _I64, _P, _P, _P, C.POINTER(_P)],
    "rsd_csr_destroy": [_P],
    "rsd_csr_info": [_P, C.POINTER(_I64), C.POINTER(_I64)],
    "rsd_csr_layout": [_P, C.POINTER(_I64), C.POINTER(_I64), C.POINTER(_I64)],
    "rsd_csr_mirrored": [_P, C.POINTER(_I64), C.POINTER(_I32)],
    "rsd_csr_values": [_P, _P, C.POINTER(_P)],
    "rsd_csr_set_values": [_P, _P, _P],
    "rsd_csr_get_values": [_P, _P, _P],
    "rsd_csr_get_pattern": [_P, _P, _P, _P],
    "rsd_spmv": [_P, _P, _P, _P],
    "rsd_csr_sync_f32": [_P, _P],
    "rsd_spmv_f32": [_P, _P, _P, _P],
    "rsd_csr_diagonal": [_P, _P, _P],
    "rsd_csr_lump": [_P, _P, _P],
    "rsd_jacobi_setup": [_P, _P, _P],
    "rsd_csr_set_launch": [_P, _I32, _I32],
    "rsd_csr_autotune": [_P, _P, C.POINTER(_I32), C.POINTER(_I32), C.POINTER(_D)],
    "rsd_measure_fp64_rate": [_P, C.POINTER(_D)],
    "rsd_solve": [_P, _P, C.POINTER(SolverConfig), _P, _P, C.POINTER(Report)],
    "rsd_cg_solve_static": [_P, _P, C.POINTER(SolverConfig), _P, _P, C.POINTER(Report)],
    "rsd_mesh_create": [_P, _I32, _I32, _I64, _I64, _P, _P, _P, C.POINTER(_P)],
    "rsd_mesh_destroy": [_P],
    "rsd_pmsh_read": [C.c_char_p, C.POINTER(PmshInfo), _P, _P, _P],
    "rsd_mesh_read_pmsh": [_P, C.c_char_p, C.POINTER(_P)],
    "rsd_heat_create": [_P, _P, C.POINTER(HeatDesc), C.POINTER(_P)],
    "rsd_heat_destroy": [_P],
    "rsd_heat_info": [_P, C.POINTER(_I64), C.POINTER(_I64)],
    "rsd_heat_dofmap": [_P, _P, _P, _P],
    "rsd_heat_matrix": [_P, C.POINTER(_P)],
    "rsd_heat_create_matrix": [_P, _P, C.POINTER(_P)],
    "rsd_heat_eval_nodal": [_P, _P, C.c_char_p, _D, _P],
    "rsd_heat_set_time": [_P, _P, _D],
    "rsd_heat_set_k_elem": [_P, _P, _P],
    "rsd_assemble_matrix": [_P, _P, _D, _D, _D, _D, _P, _P, _P],
    "rsd_assemble_vector": [_P, _P, _I32, _D, _P, _P, _P, _P],
    "rsd_apply_dirichlet_lift": [_P, _P, _D, _D, _P],
    "rsd_heat_boundary_flux": [_P, _P, _I32, _I32, _I32, _I32, _P, _P, _P, _P, _P],
    "rsd_assemble_diagonal": [_P, _P, _D, _D, _P, _P],
    "rsd_heat_solve_fem": [_P, _P, _D, C.POINTER(SolverConfig), _P, _P, C.POINTER(Report)],
    "rsd_heat_solve_fem_forms": [_P, _P, _D, _D, _D, _P, _P, C.POINTER(SolverConfig), _P, _P, C.POINTER(Report)],
    "rsd_heat_set_flux": [_P, _P, _I32, C.POINTER(C.c_char_p)],
    "rsd_apply_natural": [_P, _P, _P],
    "rsd_heat_nodal_field": [_P, _P, _I32, _P, _P, _P],
    "rsd_heat_steady": [_P, _P, C.POINTER(SolverConfig), _P, C.POINTER(Report)],
    "rsd_heat_be_step": [_P, _P, _D, C.POINTER(SolverConfig), _P, _P, C.POINTER(Report), C.POINTER(_D)],
    "rsd_heat_be_step_host": [_P, _P, _D, C.POINTER(SolverConfig), _P, C.POINTER(Report), C.POINTER(_D)],
    "rsd_heat_newton": [_P, _P, _D, _D, _I64, C.POINTER(SolverConfig), _P, C.POINTER(Report)],
    "rsd_batch_create": [_P, _I32, _P, C.POINTER(_P)],
    "rsd_batch_destroy": [_P],
    "rsd_batch_solve": [_P, _P, C.POINTER(SolverConfig), _P, _P, _P],
    "rsd_heat_forward": [_P, _P, _P, C.POINTER(SolverConfig), _P, C.POINTER(Report)],
    "rsd_heat_backward": [_P, _P, _P, _P, _P, C.POINTER(SolverConfig), _P, C.POINTER(Report)],
    "rsd_heat_transient_forward": [_P, _P, _P, _D, _D, _I64, C.POINTER(SolverConfig), _P, _P, C.POINTER(Report)],
    "rsd_heat_transient_backward": [_P, _P, _P, _D, _D, _I64, _P, _P, C.POINTER(SolverConfig), _P, C.POINTER(Report),
                                    C.POINTER(_I64)],
}


def lib():
    """Load the in-tree library (built by build.py); there is deliberately no fallback."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with residuum-solver_b200/build.py")
        L = C.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.rsd_last_error_string.restype = C.c_char_p
        L.rsd_ctx_stream.restype = _P
        _lib = L
    return _lib


def expr_check(expr):
    """Compile an expression on the host: the stack depth its device program needs (RsdError if rejected)."""
    depth = _I32()
    check(lib().rsd_expr_check(expr.encode(), C.byref(depth)))
    return depth.value


def check(rc):
    if rc != 0:
        raise RsdError(rc, lib().rsd_last_error_string().decode())


_DT = {np.float64: 8, np.float32: 4, np.int32: 4, np.int64: 8}


class Context:
    """One device + one CUDA stream (rsd_ctx)."""

    def __init__(self, device=0):
        self.h = _P()
        check(lib().rsd_ctx_create(device, C.byref(self.h)))

    def close(self):
        if self.h:
            lib().rsd_ctx_destroy(self.h)
            self.h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        check(lib().rsd_ctx_sync(self.h))

    def stream(self):
        return lib().rsd_ctx_stream(self.h)

    def profile(self, enable=True):
        """Time every launch of the library's kernel families with CUDA events (resets totals)."""
        check(lib().rsd_ctx_profile(self.h, 1 if enable else 0))

    def profile_get(self, family):
        n, ms = _I64(), _D()
        check(lib().rsd_ctx_profile_get(self.h, family.encode(), C.byref(n), C.byref(ms)))
        return n.value, ms.value

    def array(self, n, dtype=np.float64):
        return DeviceArray(self, n, dtype)

    def to_device(self, a, dtype=None):
        a = np.ascontiguousarray(a, dtype=dtype or a.dtype)
        d = DeviceArray(self, a.size, a.dtype.type)
        d.upload(a)
        return d


class DeviceArray:
    """A device allocation from rsd_alloc with numpy upload/download."""

    def __init__(self, ctx, n, dtype=np.float64):
        self.ctx, self.n, self.dtype = ctx, int(n), np.dtype(dtype).type
        self.nbytes = self.n * _DT[self.dtype]
        self.ptr = _P()
        check(lib().rsd_alloc(ctx.h, max(self.nbytes, 1), C.byref(self.ptr)))

    def __del__(self):
        try:
            if self.ptr:
                lib().rsd_free(self.ctx.h, self.ptr)
        except Exception:
            pass

    def upload(self, a):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        assert a.size == self.n
        check(lib().rsd_memcpy(self.ctx.h, self.ptr, a.ctypes.data_as(_P), self.nbytes, RSD_H2D))
        return self

    def download(self):
        out = np.empty(self.n, dtype=self.dtype)
        check(lib().rsd_memcpy(self.ctx.h, out.ctypes.data_as(_P), self.ptr, self.nbytes, RSD_D2H))
        return out

    def zero(self):
        check(lib().rsd_memset_zero(self.ctx.h, self.ptr, self.nbytes))
        return self

    def fill(self, v):
        if self.dtype == np.float64:
            check(lib().rsd_fill_f64(self.ctx.h, self.ptr, self.n, v))
        else:
            check(lib().rsd_fill_f32(self.ctx.h, self.ptr, self.n, v))
        return self


def _ptr(a):
    """Device pointer of a DeviceArray, a torch CUDA tensor (data_ptr), or a raw pointer."""
    if a is None:
        return None
    if isinstance(a, DeviceArray):
        return a.ptr
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a


class CSR:
    """rsd_csr: CSRMatrix<Real, CUDA>; 32-bit indices on the device."""

    def __init__(self, ctx, handle, owned=True):
        self.ctx, self.h, self.owned = ctx, handle, owned
        n, nnz = _I64(), _I64()
        check(lib().rsd_csr_info(self.h, C.byref(n), C.byref(nnz)))
        self.n, self.nnz = n.value, nnz.value

    @classmethod
    def from_host(cls, ctx, row_ptr, col, val=None):
        rp = np.ascontiguousarray(row_ptr, np.int64)
        cl = np.ascontiguousarray(col, np.int64)
        v = None if val is None else np.ascontiguousarray(val, np.float64)
        h = _P()
        check(lib().rsd_csr_create(ctx.h, len(rp) - 1, len(cl), rp.ctypes.data_as(_P), cl.ctypes.data_as(_P),
                                   None if v is None else v.ctypes.data_as(_P), C.byref(h)))
        return cls(ctx, h)

    def __del__(self):
        try:
            if self.owned and self.h:
                lib().rsd_csr_destroy(self.h)
        except Exception:
            pass

    def values(self):
        out = np.empty(self.nnz)
        check(lib().rsd_csr_get_values(self.ctx.h, self.h, out.ctypes.data_as(_P)))
        return out

    def set_values(self, v):
        v = np.ascontiguousarray(v, np.float64)
        check(lib().rsd_csr_set_values(self.ctx.h, self.h, v.ctypes.data_as(_P)))

    def layout(self):
        """SELL-32 slots (padding included), slices and stencil slices of the execution layout."""
        a, b, c = _I64(), _I64(), _I64()
        check(lib().rsd_csr_layout(self.h, C.byref(a), C.byref(b), C.byref(c)))
        d, e = _I64(), _I32()
        check(lib().rsd_csr_mirrored(self.h, C.byref(d), C.byref(e)))
        return {"sell_slots": a.value, "slices": b.value, "stencil_slices": c.value, "mirrored_slices": d.value,
                "mirrored_active": bool(e.value)}

    def pattern(self):
        rp = np.empty(self.n + 1, np.int64)
        col = np.empty(self.nnz, np.int64)
        check(lib().rsd_csr_get_pattern(self.ctx.h, self.h, rp.ctypes.data_as(_P), col.ctypes.data_as(_P)))
        return rp, col

    def spmv(self, x, y):
        check(lib().rsd_spmv(self.ctx.h, self.h, _ptr(x), _ptr(y)))

    def spmv_f32(self, x, y):
        check(lib().rsd_spmv_f32(self.ctx.h, self.h, _ptr(x), _ptr(y)))

    def sync_f32(self):
        check(lib().rsd_csr_sync_f32(self.ctx.h, self.h))

    def diagonal(self, d):
        check(lib().rsd_csr_diagonal(self.ctx.h, self.h, _ptr(d)))

    def lump(self, d):
        check(lib().rsd_csr_lump(self.ctx.h, self.h, _ptr(d)))

    def jacobi(self, inv_d):
        check(lib().rsd_jacobi_setup(self.ctx.h, self.h, _ptr(inv_d)))

    def set_launch(self, lanes=0, block=0):
        check(lib().rsd_csr_set_launch(self.h, lanes, block))

    def autotune(self):
        lanes, block, us = _I32(), _I32(), _D()
        check(lib().rsd_csr_autotune(self.ctx.h, self.h, C.byref(lanes), C.byref(block), C.byref(us)))
        return lanes.value, block.value, us.value


def solve(ctx, A, b, x, cfg=None, **kw):
    cfg = cfg or SolverConfig.make(**kw)
    rep = Report()
    check(lib().rsd_solve(ctx.h, A.h, C.byref(cfg), _ptr(b), _ptr(x), C.byref(rep)))
    return rep.as_dict()


class Batch:
    """rsd_batch: independent systems solved together in one persistent launch."""

    def __init__(self, ctx, mats):
        self.ctx, self.mats = ctx, list(mats)
        hs = (_P * max(len(self.mats), 1))(*[m.h for m in self.mats])
        h = _P()
        check(lib().rsd_batch_create(ctx.h, len(self.mats), hs, C.byref(h)))
        self.h = h

    def __del__(self):
        try:
            if self.h:
                lib().rsd_batch_destroy(self.h)
        except Exception:
            pass

    def solve(self, bs, xs, cfg=None, **kw):
        """bs, xs: sequences of device vectors; returns one report dict per system."""
        cfg = cfg or SolverConfig.make(**kw)
        n = len(self.mats)
        pb = (_P * max(n, 1))(*[_ptr(b) for b in bs])
        px = (_P * max(n, 1))(*[_ptr(x) for x in xs])
        reps = (Report * max(n, 1))()
        check(lib().rsd_batch_solve(self.ctx.h, self.h, C.byref(cfg), pb, px, reps))
        return [reps[i].as_dict() for i in range(n)]


def solve_static(ctx, A, b, x, cfg=None, **kw):
    """FP64 CG through rsd_cg_solve_static: no allocation, at most 262,144 rows."""
    cfg = cfg or SolverConfig.make(**kw)
    rep = Report()
    check(lib().rsd_cg_solve_static(ctx.h, A.h, C.byref(cfg), _ptr(b), _ptr(x), C.byref(rep)))
    return rep.as_dict()


class Mesh:
    """rsd_mesh from mesh::Data-layout host arrays (xyz node-major, ien element-major, rng per face)."""

    def __init__(self, ctx, nsd, order, xyz, ien, rng):
        self.ctx = ctx
        xyz = np.ascontiguousarray(xyz, np.float64)
        ien = np.ascontiguousarray(ien, np.int64)
        rng = np.ascontiguousarray(rng, np.int32)
        npe = (order + 1) ** nsd
        self.nsd, self.order, self.npe = nsd, order, npe
        self.nnodes, self.nelem = xyz.size // nsd, ien.size // npe
        self.h = _P()
        check(lib().rsd_mesh_create(ctx.h, nsd, order, self.nnodes, self.nelem, xyz.ctypes.data_as(_P),
                                    ien.ctypes.data_as(_P), rng.ctypes.data_as(_P), C.byref(self.h)))

    def __del__(self):
        try:
            if self.h:
                lib().rsd_mesh_destroy(self.h)
        except Exception:
            pass


def read_pmsh(path):
    """A PMSH mesh file on the host: (info dict, xyz, ien, rng), as MeshIO::readBinary reads it."""
    info = PmshInfo()
    check(lib().rsd_pmsh_read(path.encode(), C.byref(info), None, None, None))
    xyz = np.zeros(info.num_nodes * info.spatial_dim)
    ien = np.zeros(info.num_elements * info.nodes_per_element, np.int64)
    rng = np.zeros(info.num_elements * info.faces_per_element, np.int32)
    check(lib().rsd_pmsh_read(path.encode(), C.byref(info), xyz.ctypes.data_as(_P), ien.ctypes.data_as(_P), rng.ctypes.data_as(_P)))
    d = {k: getattr(info, k) for k, _ in PmshInfo._fields_ if k != "order"}
    d["order"] = list(info.order)[: info.num_orders]
    return d, xyz, ien, rng


class PmshMesh(Mesh):
    """A device mesh read from a PMSH file (rsd_mesh_read_pmsh)."""

    def __init__(self, ctx, path):
        info, _, _, _ = read_pmsh(path)
        self.ctx = ctx
        self.nsd, self.order = info["spatial_dim"], info["order"][0]
        self.npe = info["nodes_per_element"]
        self.nnodes, self.nelem = info["num_nodes"], info["num_elements"]
        self.h = _P()
        check(lib().rsd_mesh_read_pmsh(ctx.h, path.encode(), C.byref(self.h)))


class Heat:
    """rsd_heat: the heat problem (dof map, pattern, element loops, stages) on the device."""

    def __init__(self, ctx, mesh, nq, k_const=1.0, k_expr=None, dk_expr=None, k_elem=None, rho=1.0, cp=1.0,
                 src_expr=None, dirichlet=None, flux=None, k_tensor=None, cp_expr=None, dcp_expr=None):
        """dirichlet: {tag: expression} for boundary tags of any value >= 0; k_tensor: the conductivity's
        nsd x nsd anisotropic shape (K = k * k_tensor); cp_expr / dcp_expr: cp(T) and dcp/dT."""
        self.ctx, self.mesh = ctx, mesh
        d = HeatDesc()
        d.nq, d.k_const, d.rho, d.cp = nq, k_const, rho, cp
        d.k_expr = k_expr.encode() if k_expr else None
        d.dk_expr = dk_expr.encode() if dk_expr else None
        d.src_expr = src_expr.encode() if src_expr else None
        d.cp_expr = cp_expr.encode() if cp_expr else None
        d.dcp_expr = dcp_expr.encode() if dcp_expr else None
        ke = None if k_elem is None else np.ascontiguousarray(k_elem, np.float64)
        d.k_elem = None if ke is None else ke.ctypes.data_as(_P)
        kt = None if k_tensor is None else np.ascontiguousarray(k_tensor, np.float64).reshape(-1)
        if kt is not None and kt.size != mesh.nsd * mesh.nsd:
            raise ValueError("k_tensor must hold nsd x nsd entries")
        d.k_tensor = None if kt is None else kt.ctypes.data_as(_P)
        extra = [(tag, ex) for tag, ex in (dirichlet or {}).items() if not 0 <= tag < 6]
        for tag, ex in (dirichlet or {}).items():
            if 0 <= tag < 6:
                d.dirichlet_expr[tag] = ex.encode()
        tags = np.array([t for t, _ in extra], dtype=np.int32)
        exprs = (C.c_char_p * max(len(extra), 1))(*[ex.encode() for _, ex in extra])
        d.num_dirichlet = len(extra)
        d.dirichlet_tags = tags.ctypes.data_as(_P) if extra else None
        d.dirichlet_exprs = C.cast(exprs, _P) if extra else None
        self.h = _P()
        check(lib().rsd_heat_create(ctx.h, mesh.h, C.byref(d), C.byref(self.h)))
        n, nnz = _I64(), _I64()
        check(lib().rsd_heat_info(self.h, C.byref(n), C.byref(nnz)))
        self.n, self.nnz = n.value, nnz.value
        a = _P()
        check(lib().rsd_heat_matrix(self.h, C.byref(a)))
        self.K = CSR(ctx, a, owned=False)
        for tag, exprs in (flux or {}).items():
            self.set_flux(tag, exprs)

    def __del__(self):
        try:
            if self.h:
                lib().rsd_heat_destroy(self.h)
        except Exception:
            pass

    def dofmap(self):
        t2a = np.empty(self.mesh.nnodes, np.int32)
        a2t = np.empty(max(self.n, 1), np.int32)
        check(lib().rsd_heat_dofmap(self.ctx.h, self.h, t2a.ctypes.data_as(_P), a2t.ctypes.data_as(_P)))
        return t2a, a2t[: self.n]

    def set_time(self, t):
        check(lib().rsd_heat_set_time(self.ctx.h, self.h, t))

    def create_matrix(self):
        """A new matrix with the problem's pattern (shared) and zero values (HeatProblem::createMatrix)."""
        a = _P()
        check(lib().rsd_heat_create_matrix(self.ctx.h, self.h, C.byref(a)))
        m = CSR(self.ctx, a, owned=True)
        m._owner = self   # the pattern belongs to the problem: keep it alive
        return m

    def eval_nodal(self, expr, U, t=0.0):
        """U = expr(t, x) at the free nodes (the initial condition's Expression mode)."""
        check(lib().rsd_heat_eval_nodal(self.ctx.h, self.h, expr.encode(), t, _ptr(U)))
        return U

    def solve_fem_forms(self, b, x, c_tdiff=0.0, c_mass=0.0, c_tmass=0.0, U=None, Udot=None, cfg=None, **kw):
        """Diffusion + c_tdiff TangentDiffusion + c_mass Mass + c_tmass TangentMass without a matrix."""
        cfg = cfg or SolverConfig.make(**kw)
        rep = Report()
        check(lib().rsd_heat_solve_fem_forms(self.ctx.h, self.h, c_tdiff, c_mass, c_tmass, _ptr(U), _ptr(Udot), C.byref(cfg),
                                             _ptr(b), _ptr(x), C.byref(rep)))
        return rep.as_dict()

    def set_k_elem(self, k_dev):
        check(lib().rsd_heat_set_k_elem(self.ctx.h, self.h, _ptr(k_dev)))

    def assemble_matrix(self, c_diff=1.0, c_mass=0.0, c_tdiff=0.0, c_tmass=0.0, U=None, Udot=None, A=None):
        A = A or self.K
        check(lib().rsd_assemble_matrix(self.ctx.h, self.h, c_diff, c_mass, c_tdiff, c_tmass, _ptr(U), _ptr(Udot), A.h))
        return A

    def assemble_vector(self, which, out, coef=0.0, U=None, Udot=None, operand=None):
        check(lib().rsd_assemble_vector(self.ctx.h, self.h, which, coef, _ptr(U), _ptr(Udot), _ptr(operand), _ptr(out)))
        return out

    def lift(self, F, c_diff=1.0, c_mass=0.0):
        check(lib().rsd_apply_dirichlet_lift(self.ctx.h, self.h, c_diff, c_mass, _ptr(F)))

    def diagonal(self, d, c_diff=1.0, c_mass=0.0, U=None):
        check(lib().rsd_assemble_diagonal(self.ctx.h, self.h, c_diff, c_mass, _ptr(U), _ptr(d)))

    def set_flux(self, tag, exprs):
        """Flux boundary condition on `tag`: one expression per spatial component (None clears it)."""
        if exprs is None:
            check(lib().rsd_heat_set_flux(self.ctx.h, self.h, tag, None))
            return
        arr = (C.c_char_p * len(exprs))(*[e.encode() for e in exprs])
        check(lib().rsd_heat_set_flux(self.ctx.h, self.h, tag, arr))

    def nodal_field(self, U, field="heat_flux"):
        """Nodal recovery of the heat flux (nnodes x nsd) or the conductivity (nnodes) from U."""
        f = {"heat_flux": 0, "conductivity": 1}[field]
        nc = self.mesh.nsd if f == 0 else 1
        out = self.ctx.array(self.mesh.nnodes * nc)
        scratch = self.ctx.array(self.mesh.nnodes)
        check(lib().rsd_heat_nodal_field(self.ctx.h, self.h, f, _ptr(U), _ptr(out), _ptr(scratch)))
        a = out.download()
        return a.reshape(-1, nc) if nc > 1 else a

    def boundary_flux(self, tags, U, Udot=None, method="weak", reduction="integral", transient=False):
        """HeatFlux monitors per boundary tag at the current time: (values, measures)."""
        tg = np.ascontiguousarray(list(tags), np.int32)
        vals, meas = np.zeros(len(tg)), np.zeros(len(tg))
        check(lib().rsd_heat_boundary_flux(self.ctx.h, self.h, {"weak": 0, "strong": 1}[method],
                                           {"integral": 0, "average": 1}[reduction], 1 if transient else 0, len(tg),
                                           tg.ctypes.data_as(_P), _ptr(U), _ptr(Udot), vals.ctypes.data_as(_P),
                                           meas.ctypes.data_as(_P)))
        return vals, meas

    def apply_natural(self, F):
        check(lib().rsd_apply_natural(self.ctx.h, self.h, _ptr(F)))

    def solve_fem(self, b, x, c_mass=0.0, cfg=None, **kw):
        """(Diffusion + c_mass Mass) x = b without a matrix: the LinearSolverRunner the reference builds
        for operator type `fem` (FEMOperator), CG or GMRES(m) + Jacobi in FP64; x holds the initial guess."""
        cfg = cfg or SolverConfig.make(**kw)
        rep = Report()
        check(lib().rsd_heat_solve_fem(self.ctx.h, self.h, c_mass, C.byref(cfg), _ptr(b), _ptr(x), C.byref(rep)))
        return rep.as_dict()

    def steady(self, U, cfg=None, **kw):
        cfg = cfg or SolverConfig.make(**kw)
        rep = Report()
        check(lib().rsd_heat_steady(self.ctx.h, self.h, C.byref(cfg), _ptr(U), C.byref(rep)))
        return rep.as_dict()

    def be_step(self, dt, U, Uprev, cfg=None, **kw):
        cfg = cfg or SolverConfig.make(**kw)
        rep, res = Report(), _D()
        check(lib().rsd_heat_be_step(self.ctx.h, self.h, dt, C.byref(cfg), _ptr(U), _ptr(Uprev), C.byref(rep), C.byref(res)))
        d = rep.as_dict()
        d["residualNorm"] = res.value
        return d

    def be_step_host(self, dt, U_host, cfg=None, **kw):
        """The step with the state in host memory: U_host (a C-contiguous float64 numpy array or CPU
        torch tensor, pinned for full-speed copies) holds the state on entry and the new state on
        return."""
        cfg = cfg or SolverConfig.make(**kw)
        rep, res = Report(), _D()
        if hasattr(U_host, "ctypes"):
            if U_host.dtype != np.float64 or not U_host.flags["C_CONTIGUOUS"] or U_host.size != self.n:
                raise ValueError("U_host must be a C-contiguous float64 array of the problem's size")
            ptr = U_host.ctypes.data_as(_P)
        else:
            if U_host.dtype != __import__("torch").float64 or U_host.is_cuda or U_host.numel() != self.n:
                raise ValueError("U_host must be a float64 CPU tensor of the problem's size")
            ptr = C.c_void_p(U_host.data_ptr())
        check(lib().rsd_heat_be_step_host(self.ctx.h, self.h, dt, C.byref(cfg), ptr, C.byref(rep), C.byref(res)))
        d = rep.as_dict()
        d["residualNorm"] = res.value
        return d

    def forward(self, theta, T, cfg=None, **kw):
        """Adjoint pair, forward: k_e = k_const exp(theta_e), solve K(theta) T = F (T: warm start in,
        solution out).  theta, T: device arrays (DeviceArray or anything with .ptr / data_ptr())."""
        cfg = cfg or SolverConfig.make(**kw)
        rep = Report()
        check(lib().rsd_heat_forward(self.ctx.h, self.h, _ptr(theta), C.byref(cfg), _ptr(T), C.byref(rep)))
        return rep.as_dict()

    def backward(self, theta, T, dJdT, dJdtheta, cfg=None, **kw):
        """Adjoint pair, backward: solve K lambda = dJ/dT and write dJ/dtheta per element."""
        cfg = cfg or SolverConfig.make(**kw)
        rep = Report()
        check(lib().rsd_heat_backward(self.ctx.h, self.h, _ptr(theta), _ptr(T), _ptr(dJdT), C.byref(cfg),
                                      _ptr(dJdtheta), C.byref(rep)))
        return rep.as_dict()

    def transient_forward(self, theta, U0, U, t0, dt, nsteps, cfg=None, **kw):
        """Transient pair, forward: U = the state after nsteps Backward-Euler steps from U0 with
        k_e = k_const exp(theta_e)."""
        cfg = cfg or SolverConfig.make(**kw)
        rep = Report()
        check(lib().rsd_heat_transient_forward(self.ctx.h, self.h, _ptr(theta), t0, dt, nsteps, C.byref(cfg), _ptr(U0),
                                               _ptr(U), C.byref(rep)))
        return rep.as_dict()

    def transient_backward(self, theta, U0, dJdU, dJdtheta, t0, dt, nsteps, cfg=None, **kw):
        """Transient pair, backward: dJ/dtheta of a terminal objective J(U_N) (dJdU given) by the
        discrete adjoint, the forward states replayed from checkpoints; returns the report with
        "states_held", the states kept at once."""
        cfg = cfg or SolverConfig.make(**kw)
        rep, held = Report(), _I64()
        check(lib().rsd_heat_transient_backward(self.ctx.h, self.h, _ptr(theta), t0, dt, nsteps, _ptr(U0), _ptr(dJdU),
                                                C.byref(cfg), _ptr(dJdtheta), C.byref(rep), C.byref(held)))
        d = rep.as_dict()
        d["states_held"] = held.value
        return d

    def newton(self, U, abs_tol=1e-10, rel_tol=1e-10, max_iters=50, cfg=None, **kw):
        cfg = cfg or SolverConfig.make(type=GMRES, **kw)
        rep = Report()
        check(lib().rsd_heat_newton(self.ctx.h, self.h, abs_tol, rel_tol, max_iters, C.byref(cfg), _ptr(U), C.byref(rep)))
        return rep.as_dict()
