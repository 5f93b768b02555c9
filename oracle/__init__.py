"""Test infrastructure, not product code.

ctypes front ends for the two CPU checkers of the CUDA backend:

* ``Oracle`` - the plain-C restatement in ``rsd_oracle.c`` (``_build/librsd_oracle.so``);
* ``Reference`` - the Residuum reference templates compiled unmodified through
  ``ref_harness.cpp`` (``_ref/libresiduum_ref.so``), present wherever ``build()`` could see the
  reference checkout.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this package.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "librsd_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libresiduum_ref.so")

_P = C.c_void_p
_D = C.c_double
_I32 = C.c_int32
_I64 = C.c_int64


def build(ref_root=None):
    """Compile the restatement and, when `ref_root` names the reference checkout, the reference
    harness from the sources there."""
    targets = ["all"]
    args = []
    if ref_root:
        if not os.path.isdir(ref_root):
            raise FileNotFoundError(f"reference checkout {ref_root!r} does not exist")
        targets.append("ref")
        args.append("REF=" + ref_root)
    subprocess.run(["make", "-s", "-C", HERE] + args + targets, check=True)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


class Report(C.Structure):
    _fields_ = [("converged", _I32), ("iterations", _I64), ("initialResidual", _D),
                ("finalResidual", _D), ("finalResidualRel", _D)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


# ---------------------------------------------------------------------------------------------
# restatement
# ---------------------------------------------------------------------------------------------
class _Mesh(C.Structure):
    _fields_ = [("nsd", _I32), ("order", _I32), ("nnodes", _I64), ("nelem", _I64), ("npe", _I32),
                ("nfaces", _I32), ("xyz", C.POINTER(_D)), ("ien", C.POINTER(_I64)), ("rng", C.POINTER(_I32))]


class _Model(C.Structure):
    _fields_ = [("nq", _I32), ("k_expr", C.c_char_p), ("dk_expr", C.c_char_p), ("k_const", _D),
                ("k_elem", _P), ("rho", _D), ("cp", _D), ("src_expr", C.c_char_p), ("bc_expr", C.c_char_p * 6)]


_olib = None


def oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle library missing: run oracle.build() (make -C oracle)")
        L = C.CDLL(ORACLE_SO)
        L.ro_mesh_block.argtypes = [_I32, _P, _P, _P, _I32, C.POINTER(_Mesh)]
        L.ro_mesh_free.argtypes = [C.POINTER(_Mesh)]
        L.ro_problem_create.argtypes = [C.POINTER(_Mesh), C.POINTER(_Model)]
        L.ro_problem_create.restype = _P
        L.ro_problem_destroy.argtypes = [_P]
        L.ro_last_error.restype = C.c_char_p
        L.ro_num_free.argtypes = [_P]; L.ro_num_free.restype = _I64
        L.ro_nnz.argtypes = [_P]; L.ro_nnz.restype = _I64
        L.ro_dofmap.argtypes = [_P, _P, _P, _P]
        L.ro_pattern.argtypes = [_P, _P, _P]
        L.ro_set_time.argtypes = [_P, _D]
        L.ro_bc_node_values.argtypes = [_P, _P]
        L.ro_assemble_matrix.argtypes = [_P, _D, _D, _D, _D, _P, _P, _P]
        L.ro_assemble_vector.argtypes = [_P, _I32, _D, _P, _P, _P, _P]
        L.ro_lift.argtypes = [_P, _D, _D, _P]
        L.ro_diagonal.argtypes = [_P, _D, _D, _P, _P]
        L.ro_adjoint_gradient.argtypes = [_P, _P, _P, _P]
        L.ro_spmv.argtypes = [_I64, _P, _P, _P, _P, _P]
        L.ro_csr_solve.argtypes = [_I32, _I32, _I64, _P, _P, _P, _P, _P, _D, _I64, _I64, C.POINTER(Report)]
        L.ro_steady.argtypes = [_P, _I32, _I32, _D, _I64, _I64, _P, C.POINTER(Report)]
        L.ro_backward_euler.argtypes = [_P, _D, _I64, _I32, _I32, _D, _I64, _I64, _P, _P, _P]
        L.ro_newton.argtypes = [_P, _D, _D, _I64, _I32, _I32, _D, _I64, _I64, _P, C.POINTER(Report)]
        L.ro_expr_eval.argtypes = [C.c_char_p, _D, _D, _D, _D, _D, C.POINTER(_D)]
        L.ro_fem_solve.argtypes = [_P, _D, _I32, _P, _P, _D, _I64, C.POINTER(Report)]
        L.ro_set_operator.argtypes = [_P, _I32]
        L.ro_set_flux.argtypes = [_P, _I32, C.POINTER(C.c_char_p)]
        L.ro_natural.argtypes = [_P, _P]
        L.ro_nodal_field.argtypes = [_P, _I32, _P, _P]
        _olib = L
    return _olib


def expr_eval(src, t=0.0, x=0.0, y=0.0, z=0.0, T=0.0):
    out = _D()
    if oracle_lib().ro_expr_eval(src.encode(), t, x, y, z, T, C.byref(out)):
        raise ValueError(oracle_lib().ro_last_error().decode())
    return out.value


class BlockMesh:
    """BlockMesh2D/3D through the restatement; arrays copied out as numpy."""

    def __init__(self, nsd, nel, lo, hi, order):
        L = oracle_lib()
        self._m = _Mesh()
        nel = np.asarray(list(nel) + [1] * (3 - len(nel)), dtype=np.int32)
        lo = np.asarray(list(lo) + [0.0] * (3 - len(lo)), dtype=np.float64)
        hi = np.asarray(list(hi) + [0.0] * (3 - len(hi)), dtype=np.float64)
        if L.ro_mesh_block(nsd, _ptr(nel), _ptr(lo), _ptr(hi), order, C.byref(self._m)):
            raise ValueError(L.ro_last_error().decode())
        m = self._m
        self.nsd, self.order, self.npe, self.nfaces = m.nsd, m.order, m.npe, m.nfaces
        self.nnodes, self.nelem = m.nnodes, m.nelem
        self.xyz = np.ctypeslib.as_array(m.xyz, shape=(m.nnodes * m.nsd,)).copy()
        self.ien = np.ctypeslib.as_array(m.ien, shape=(m.nelem * m.npe,)).copy()
        self.rng = np.ctypeslib.as_array(m.rng, shape=(m.nelem * m.nfaces,)).copy()

    def __del__(self):
        try:
            oracle_lib().ro_mesh_free(C.byref(self._m))
        except Exception:
            pass


class Oracle:
    """The restatement for one mesh + model: dof map, pattern, element loops, solvers, stages."""

    def __init__(self, mesh, nq, k_const=1.0, k_expr=None, dk_expr=None, k_elem=None, rho=1.0, cp=1.0,
                 src_expr=None, bc=None, flux=None):
        L = oracle_lib()
        self.mesh = mesh
        self._kelem = None if k_elem is None else _f64(k_elem)
        md = _Model()
        md.nq = nq
        md.k_expr = k_expr.encode() if k_expr else None
        md.dk_expr = dk_expr.encode() if dk_expr else None
        md.k_const = k_const
        md.k_elem = _ptr(self._kelem)
        md.rho, md.cp = rho, cp
        md.src_expr = src_expr.encode() if src_expr else None
        for tag, ex in (bc or {}).items():
            md.bc_expr[tag] = ex.encode()
        self._model = md
        self.h = L.ro_problem_create(C.byref(mesh._m), C.byref(md))
        if not self.h:
            raise ValueError(L.ro_last_error().decode())
        self.n = L.ro_num_free(self.h)
        self.nnz = L.ro_nnz(self.h)
        for tag, exprs in (flux or {}).items():
            arr = (C.c_char_p * len(exprs))(*[e.encode() for e in exprs])
            if L.ro_set_flux(self.h, tag, arr):
                raise ValueError(L.ro_last_error().decode())

    def __del__(self):
        try:
            oracle_lib().ro_problem_destroy(self.h)
        except Exception:
            pass

    def dofmap(self):
        t2a = np.zeros(self.mesh.nnodes, np.int32)
        a2t = np.zeros(max(self.n, 1), np.int32)
        ctag = np.zeros(self.mesh.nnodes, np.int32)
        oracle_lib().ro_dofmap(self.h, _ptr(t2a), _ptr(a2t), _ptr(ctag))
        return t2a, a2t[: self.n], ctag

    def pattern(self):
        rp = np.zeros(self.n + 1, np.int64)
        col = np.zeros(max(self.nnz, 1), np.int64)
        oracle_lib().ro_pattern(self.h, _ptr(rp), _ptr(col))
        return rp, col[: self.nnz]

    def set_time(self, t):
        oracle_lib().ro_set_time(self.h, t)

    def bc_node_values(self):
        g = np.zeros(self.mesh.nnodes)
        oracle_lib().ro_bc_node_values(self.h, _ptr(g))
        return g

    def assemble_matrix(self, c_diff=1.0, c_mass=0.0, c_tdiff=0.0, c_tmass=0.0, U=None, Udot=None):
        val = np.zeros(self.nnz)
        oracle_lib().ro_assemble_matrix(self.h, c_diff, c_mass, c_tdiff, c_tmass, _ptr(_f64(U)), _ptr(_f64(Udot)), _ptr(val))
        return val

    def assemble_vector(self, which, coef=0.0, U=None, Udot=None, operand=None):
        out = np.zeros(self.n)
        U, Udot, operand = _f64(U), _f64(Udot), _f64(operand)
        oracle_lib().ro_assemble_vector(self.h, which, coef, _ptr(U), _ptr(Udot), _ptr(operand), _ptr(out))
        return out

    def lift(self, F, c_diff=1.0, c_mass=0.0):
        F = np.array(F, dtype=np.float64)
        oracle_lib().ro_lift(self.h, c_diff, c_mass, _ptr(F))
        return F

    def nodal_field(self, U, field="heat_flux"):
        """Nodal recovery (SimpleAverageRecovery) of the heat flux (nnodes x nsd) or the conductivity."""
        f = {"heat_flux": 0, "conductivity": 1}[field]
        nc = self.mesh.nsd if f == 0 else 1
        out = np.zeros(self.mesh.nnodes * nc)
        oracle_lib().ro_nodal_field(self.h, f, _ptr(_f64(U)), _ptr(out))
        return out.reshape(-1, nc) if nc > 1 else out

    def natural(self, F):
        """F plus the flux boundary integrals (applyNaturalBCs) at the current time."""
        F = np.array(F, dtype=np.float64)
        oracle_lib().ro_natural(self.h, _ptr(F))
        return F

    def diagonal(self, c_diff=1.0, c_mass=0.0, U=None):
        d = np.zeros(self.n)
        oracle_lib().ro_diagonal(self.h, c_diff, c_mass, _ptr(_f64(U)), _ptr(d))
        return d

    def adjoint_gradient(self, T, lam):
        g = np.zeros(self.mesh.nelem)
        oracle_lib().ro_adjoint_gradient(self.h, _ptr(_f64(T)), _ptr(_f64(lam)), _ptr(g))
        return g

    def set_operator(self, op):
        """Operator of the stages' linear solves: "csr" (assembled matrix) or "fem" (matrix-free, CG)."""
        oracle_lib().ro_set_operator(self.h, {"csr": 0, "fem": 1}[op])

    def fem_solve(self, b, x0, coef=0.0, precond=1, tol=1e-10, maxit=1000):
        """(Diffusion + coef Mass) x = b by CG over element-pass products (FEMOperator)."""
        x = np.array(x0, dtype=np.float64)
        rep = Report()
        oracle_lib().ro_fem_solve(self.h, coef, precond, _ptr(np.asarray(b, np.float64)), _ptr(x), tol, maxit, C.byref(rep))
        return x, rep.as_dict()

    def steady(self, solver=0, precond=1, tol=1e-10, maxit=1000, krylov=30, U=None):
        U = np.zeros(self.n) if U is None else np.array(U, dtype=np.float64)
        rep = Report()
        oracle_lib().ro_steady(self.h, solver, precond, tol, maxit, krylov, _ptr(U), C.byref(rep))
        return U, rep.as_dict()

    def backward_euler(self, dt, nsteps, U0, solver=0, precond=1, tol=1e-8, maxit=1000, krylov=30):
        U = np.array(U0, dtype=np.float64)
        res = np.zeros(nsteps)
        its = np.zeros(nsteps, np.int64)
        rc = oracle_lib().ro_backward_euler(self.h, dt, nsteps, solver, precond, tol, maxit, krylov, _ptr(U), _ptr(res), _ptr(its))
        return U, res, its, rc

    def newton(self, abs_tol=1e-10, rel_tol=1e-10, maxit=50, solver=1, precond=1, tol=1e-12, lin_maxit=1000,
               krylov=30, U=None):
        U = np.zeros(self.n) if U is None else np.array(U, dtype=np.float64)
        rep = Report()
        oracle_lib().ro_newton(self.h, abs_tol, rel_tol, maxit, solver, precond, tol, lin_maxit, krylov, _ptr(U), C.byref(rep))
        return U, rep.as_dict()


def spmv(rowPtr, col, val, x):
    rowPtr = np.ascontiguousarray(rowPtr, np.int64)
    col = np.ascontiguousarray(col, np.int64)
    y = np.zeros(len(rowPtr) - 1)
    oracle_lib().ro_spmv(len(rowPtr) - 1, _ptr(rowPtr), _ptr(col), _ptr(_f64(val)), _ptr(_f64(x)), _ptr(y))
    return y


def csr_solve(rowPtr, col, val, b, x0=None, solver=0, precond=1, tol=1e-10, maxit=1000, krylov=30):
    rowPtr = np.ascontiguousarray(rowPtr, np.int64)
    col = np.ascontiguousarray(col, np.int64)
    n = len(rowPtr) - 1
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    rep = Report()
    oracle_lib().ro_csr_solve(solver, precond, n, _ptr(rowPtr), _ptr(col), _ptr(_f64(val)), _ptr(_f64(b)), _ptr(x),
                              tol, maxit, krylov, C.byref(rep))
    return x, rep.as_dict()


# ---------------------------------------------------------------------------------------------
# reference harness
# ---------------------------------------------------------------------------------------------
class _RefDesc(C.Structure):
    _fields_ = [("nsd", _I32), ("order", _I32), ("nq", _I32), ("nx", _I32), ("ny", _I32), ("nz", _I32),
                ("lo", _D * 3), ("hi", _D * 3), ("ess_mask", _I32), ("bc_kind", _I32), ("bc_val", _D * 6),
                ("src_kind", _I32), ("src_c", _D), ("k_a", _D), ("k_b", _D), ("rho", _D), ("cp", _D),
                ("k_elem", _P)]


_rlib = None


def reference_available():
    return os.path.exists(REF_SO)


def ref_lib():
    global _rlib
    if _rlib is None:
        # The harness instantiates std::num_put facets itself; loaded RTLD_LOCAL its facet ids
        # would differ from libstdc++'s and the reference's ostringstream formatting
        # (solver/linear/LinearSolverFactory.hpp:44-46) would index the wrong facet.  Putting
        # libstdc++ in the global scope first makes every facet id resolve to one definition.
        C.CDLL("libstdc++.so.6", mode=C.RTLD_GLOBAL)
        L = C.CDLL(REF_SO)
        L.ref_create.argtypes = [C.POINTER(_RefDesc)]; L.ref_create.restype = _P
        L.ref_destroy.argtypes = [_P]
        L.ref_last_error.restype = C.c_char_p
        for f in ("ref_num_nodes", "ref_num_elems", "ref_num_free", "ref_nnz"):
            getattr(L, f).argtypes = [_P]; getattr(L, f).restype = _I64
        L.ref_dofmap.argtypes = [_P, _P, _P]
        L.ref_mesh.argtypes = [_P, _P, _P, _P]
        L.ref_pattern.argtypes = [_P, _P, _P]
        L.ref_assemble_matrix.argtypes = [_P, C.c_int, _D, _P, _P, _P]
        L.ref_assemble_vector.argtypes = [_P, C.c_int, _D, _P, _P, _P, _P]
        L.ref_lift.argtypes = [_P, C.c_int, _D, _P]
        L.ref_diagonal.argtypes = [_P, C.c_int, _D, _P, _P]
        L.ref_steady.argtypes = [_P, C.c_int, C.c_int, _D, _I64, _I64, _P, C.POINTER(Report)]
        L.ref_newton.argtypes = [_P, _D, _D, _I64, C.c_int, C.c_int, _D, _I64, _I64, _P, C.POINTER(Report)]
        L.ref_backward_euler.argtypes = [_P, _D, _I64, C.c_int, C.c_int, _D, _I64, _I64, _P, _P, _P]
        L.ref_adjoint_gradient.argtypes = [_P, _P, _P, _P]
        L.ref_csr_solve.argtypes = [C.c_int, C.c_int, _I64, _P, _P, _P, _P, _P, _D, _I64, _I64, C.POINTER(Report)]
        L.ref_spmv.argtypes = [_I64, _P, _P, _P, _P, _P]
        L.ref_set_operator.argtypes = [_P, C.c_int]
        L.ref_nodal_field.argtypes = [_P, C.c_int, _P, _P]
        L.ref_boundary_flux.argtypes = [_P, C.c_int, C.c_int, C.c_int, C.c_int, _P, _P, _P, _P]
        _rlib = L
    return _rlib


class Reference:
    """The reference's own templates for one block mesh (closed-form models, see ref_harness.cpp).

    bc_kind 0: constant per essential tag (bc_val); 1: g = x; 2: g = (1-x)(1-y).
    src_kind 0: f = src_c; 1: f = src_c * x*y(*z).  k(T) = k_a + k_b*T.
    """

    FORMSETS = {"K": 0, "K+cM": 1, "K+KT": 2, "J_BE": 3, "M": 4}

    def __init__(self, nsd, order, nq, nel, lo, hi, ess_tags, bc_kind=0, bc_val=None, src_kind=0, src_c=0.0,
                 k_a=1.0, k_b=0.0, rho=1.0, cp=1.0, k_elem=None):
        L = ref_lib()
        d = _RefDesc()
        d.nsd, d.order, d.nq = nsd, order, nq
        nel = list(nel) + [1] * (3 - len(nel))
        d.nx, d.ny, d.nz = nel
        for i in range(nsd):
            d.lo[i], d.hi[i] = lo[i], hi[i]
        d.ess_mask = sum(1 << t for t in ess_tags)
        d.bc_kind = bc_kind
        for t, v in (bc_val or {}).items():
            d.bc_val[t] = v
        d.src_kind, d.src_c = src_kind, src_c
        d.k_a, d.k_b, d.rho, d.cp = k_a, k_b, rho, cp
        self._kelem = None if k_elem is None else _f64(k_elem)
        d.k_elem = _ptr(self._kelem)
        self.h = L.ref_create(C.byref(d))
        if not self.h:
            raise ValueError(L.ref_last_error().decode())
        self.nsd = nsd
        self.nnodes = L.ref_num_nodes(self.h)
        self.nelem = L.ref_num_elems(self.h)
        self.n = L.ref_num_free(self.h)
        self._nnz = None

    def __del__(self):
        try:
            ref_lib().ref_destroy(self.h)
        except Exception:
            pass

    @property
    def nnz(self):
        if self._nnz is None:
            self._nnz = ref_lib().ref_nnz(self.h)
        return self._nnz

    def dofmap(self):
        t2a = np.zeros(self.nnodes, np.int32)
        a2t = np.zeros(max(self.n, 1), np.int32)
        ref_lib().ref_dofmap(self.h, _ptr(t2a), _ptr(a2t))
        return t2a, a2t[: self.n]

    def pattern(self):
        rp = np.zeros(self.n + 1, np.int64)
        col = np.zeros(max(self.nnz, 1), np.int64)
        ref_lib().ref_pattern(self.h, _ptr(rp), _ptr(col))
        return rp, col[: self.nnz]

    def assemble_matrix(self, formset="K", c=0.0, U=None, Udot=None):
        val = np.zeros(self.nnz)
        ref_lib().ref_assemble_matrix(self.h, self.FORMSETS[formset], c, _ptr(_f64(U)), _ptr(_f64(Udot)), _ptr(val))
        return val

    def assemble_vector(self, which, coef=0.0, U=None, Udot=None, operand=None):
        out = np.zeros(self.n)
        U, Udot, operand = _f64(U), _f64(Udot), _f64(operand)
        ref_lib().ref_assemble_vector(self.h, which, coef, _ptr(U), _ptr(Udot), _ptr(operand), _ptr(out))
        return out

    def lift(self, F, formset="K", c=0.0):
        F = np.array(F, dtype=np.float64)
        ref_lib().ref_lift(self.h, self.FORMSETS[formset], c, _ptr(F))
        return F

    def diagonal(self, formset="K", c=0.0, U=None):
        d = np.zeros(self.n)
        ref_lib().ref_diagonal(self.h, self.FORMSETS[formset], c, _ptr(_f64(U)), _ptr(d))
        return d

    def nodal_field(self, U, field="heat_flux"):
        """The reference's QuantityEvaluator::evaluateNodalField (SimpleAverageRecovery)."""
        f = {"heat_flux": 0, "conductivity": 1}[field]
        nc = self.nsd if f == 0 else 1
        out = np.zeros(self.nnodes * nc)
        ref_lib().ref_nodal_field(self.h, f, _ptr(_f64(U)), _ptr(out))
        return out.reshape(-1, nc) if nc > 1 else out

    def set_operator(self, op):
        """LinearSolverConfig::OperatorType of the stages' linear solves: "csr" or "fem" (FEMOperator)."""
        ref_lib().ref_set_operator(self.h, {"csr": 0, "fem": 1}[op])

    def steady(self, solver=0, precond=1, tol=1e-10, maxit=1000, krylov=30, U=None):
        U = np.zeros(self.n) if U is None else np.array(U, dtype=np.float64)
        rep = Report()
        ref_lib().ref_steady(self.h, solver, precond, tol, maxit, krylov, _ptr(U), C.byref(rep))
        return U, rep.as_dict()

    def newton(self, abs_tol=1e-10, rel_tol=1e-10, maxit=50, solver=1, precond=1, tol=1e-12, lin_maxit=1000,
               krylov=30, U=None):
        U = np.zeros(self.n) if U is None else np.array(U, dtype=np.float64)
        rep = Report()
        ref_lib().ref_newton(self.h, abs_tol, rel_tol, maxit, solver, precond, tol, lin_maxit, krylov, _ptr(U), C.byref(rep))
        return U, rep.as_dict()

    def backward_euler(self, dt, nsteps, U0, solver=0, precond=1, tol=1e-8, maxit=1000, krylov=30, stats=False):
        """BackwardEulerRunner over BackwardEulerStage; with stats=True also returns per-step
        (step seconds, solve seconds, CG iterations) measured around the reference calls."""
        U = np.array(U0, dtype=np.float64)
        res = np.zeros(nsteps)
        st = np.zeros(3 * nsteps)
        rc = ref_lib().ref_backward_euler(self.h, dt, nsteps, solver, precond, tol, maxit, krylov, _ptr(U), _ptr(res), _ptr(st))
        if stats:
            return U, res, rc, st.reshape(nsteps, 3)
        return U, res, rc

    def adjoint_gradient(self, T, lam):
        g = np.zeros(self.nelem)
        ref_lib().ref_adjoint_gradient(self.h, _ptr(_f64(T)), _ptr(_f64(lam)), _ptr(g))
        return g

    def boundary_flux(self, tags, U, Udot=None, method="weak", reduction="integral", transient=False):
        """The reference's HeatFlux monitor groups (BoundaryReactionMonitorGroup for "weak",
        BoundaryQuadratureMonitorGroup with HeatFluxIntegrand for "strong"), one combination per tag."""
        tg = np.ascontiguousarray(list(tags), np.int32)
        out = np.zeros(len(tg))
        Udot = np.zeros(self.n) if Udot is None else Udot
        if ref_lib().ref_boundary_flux(self.h, {"weak": 0, "strong": 1}[method], {"integral": 0, "average": 1}[reduction],
                                       1 if transient else 0, len(tg), _ptr(tg), _ptr(_f64(U)), _ptr(_f64(Udot)), _ptr(out)):
            raise RuntimeError(ref_lib().ref_last_error().decode())
        return out


def ref_csr_solve(rowPtr, col, val, b, x0=None, solver=0, precond=1, tol=1e-10, maxit=1000, krylov=30):
    rowPtr = np.ascontiguousarray(rowPtr, np.int64)
    col = np.ascontiguousarray(col, np.int64)
    n = len(rowPtr) - 1
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    rep = Report()
    ref_lib().ref_csr_solve(solver, precond, n, _ptr(rowPtr), _ptr(col), _ptr(_f64(val)), _ptr(_f64(b)), _ptr(x),
                            tol, maxit, krylov, C.byref(rep))
    return x, rep.as_dict()


# ---------------------------------------------------------------------------------------------
# the reference's application layer (ref_problem.cpp): HeatProblem<CPU, HeatEquation> from a config
# ---------------------------------------------------------------------------------------------
class _RefpDesc(C.Structure):
    _fields_ = [("nsd", _I32), ("order", _I32), ("nq", _I32), ("nel", _I32 * 3), ("lo", _D * 3), ("hi", _D * 3),
                ("tag_map", _I32 * 6), ("k_type", _I32), ("k_value", _D), ("k_tensor", _D * 9),
                ("k_expr", C.c_char_p), ("dk_expr", C.c_char_p), ("rho", _D), ("cp_type", _I32), ("cp_value", _D),
                ("cp_expr", C.c_char_p), ("dcp_expr", C.c_char_p), ("source", C.c_char_p), ("initial", C.c_char_p),
                ("nbc", _I32), ("bc_tag", _I32 * 16), ("bc_flux", _I32 * 16), ("bc_expr", (C.c_char_p * 3) * 16),
                ("transient", _I32), ("nonlinear", _I32), ("nl_abs", _D), ("nl_rel", _D), ("nl_maxit", _I64),
                ("lin_type", _I32), ("precond", _I32), ("op_type", _I32), ("lin_tol", _D), ("lin_maxit", _I64),
                ("krylov", _I64), ("t0", _D), ("tf", _D), ("dt", _D)]


_refp_bound = False


def _refp_lib():
    global _refp_bound
    L = ref_lib()
    if not _refp_bound:
        L.refp_create.argtypes = [C.POINTER(_RefpDesc)]; L.refp_create.restype = _P
        L.refp_destroy.argtypes = [_P]
        L.refp_last_error.restype = C.c_char_p
        L.refp_num_free.argtypes = [_P]; L.refp_num_free.restype = _I64
        L.refp_num_nodes.argtypes = [_P]; L.refp_num_nodes.restype = _I64
        L.refp_nnz.argtypes = [_P]; L.refp_nnz.restype = _I64
        L.refp_mesh.argtypes = [_P, _P, _P]
        L.refp_dofmap.argtypes = [_P, _P]
        L.refp_run.argtypes = [_P, _P]
        L.refp_pattern.argtypes = [_P, _P, _P]
        L.refp_assemble_matrix.argtypes = [_P, C.c_int, _D, _D, _P, _P, _P]
        L.refp_assemble_vector.argtypes = [_P, C.c_int, _D, _P, _P, _P]
        L.refp_write_pmsh.argtypes = [C.POINTER(_RefpDesc), C.c_char_p]
        _refp_bound = True
    return L


class RefProblem:
    """The reference's HeatProblem<CPU, HeatEquation<nsd, nsd, Quad|Hex>> on a block mesh, built from
    a HeatConfig with its own models, and solved by its own stages and drivers.

    conductivity: ("constant", k) | ("anisotropic", tensor) | ("k(T)", k_expr, dk_expr)
                  | ("k(T) tensor", tensor, k_expr, dk_expr)
    specific_heat: ("constant", cp) | ("cp(T)", cp_expr, dcp_expr)   (transient runs only)
    bcs: list of (tag, "value", expr) or (tag, "flux", [expr per component])
    tag_map: {block tag: new tag} renumbers the block mesh's boundary tags
    solver: dict(type "cg"|"gmres", precond "jacobi"|"identity", operator "csr"|"fem", tol, maxit, krylov,
                 newton=(abs, rel, maxit) or None, transient=(t0, tf, dt) or None)
    """

    def __init__(self, nsd, order, nq, nel, lo, hi, conductivity=("constant", 1.0), rho=1.0,
                 specific_heat=("constant", 1.0), source="0", initial="0", bcs=(), tag_map=None, solver=None):
        L = _refp_lib()
        d = _RefpDesc()
        self._keep = []

        def s(x):
            if x is None:
                return None
            b = x.encode()
            self._keep.append(b)
            return b
        d.nsd, d.order, d.nq = nsd, order, nq
        nel = list(nel) + [1] * (3 - len(nel))
        for i in range(3):
            d.nel[i] = nel[i]
        for i in range(nsd):
            d.lo[i], d.hi[i] = lo[i], hi[i]
        for t in range(6):
            d.tag_map[t] = (tag_map or {}).get(t, -1)
        kind = conductivity[0]
        d.k_type = {"constant": 0, "anisotropic": 1, "k(T)": 2, "k(T) tensor": 3}[kind]
        if kind == "constant":
            d.k_value = conductivity[1]
        if kind in ("anisotropic", "k(T) tensor"):
            t = np.asarray(conductivity[1], dtype=np.float64).reshape(nsd, nsd)
            for i in range(nsd * nsd):
                d.k_tensor[i] = t.flat[i]
        if kind in ("k(T)", "k(T) tensor"):
            d.k_expr, d.dk_expr = s(conductivity[-2]), s(conductivity[-1])
        d.rho = rho
        if specific_heat[0] == "constant":
            d.cp_type, d.cp_value = 0, specific_heat[1]
        else:
            d.cp_type, d.cp_expr, d.dcp_expr = 1, s(specific_heat[1]), s(specific_heat[2])
        d.source, d.initial = s(source), s(initial)
        d.nbc = len(bcs)
        for b, (tag, kind, ex) in enumerate(bcs):
            d.bc_tag[b] = tag
            d.bc_flux[b] = 1 if kind == "flux" else 0
            exprs = [ex] if kind != "flux" else list(ex)
            for i, e in enumerate(exprs):
                d.bc_expr[b][i] = s(e)
        sv = dict(type="cg", precond="jacobi", operator="csr", tol=1e-10, maxit=1000, krylov=30, newton=None, transient=None)
        sv.update(solver or {})
        d.lin_type = 1 if sv["type"] == "gmres" else 0
        d.precond = 1 if sv["precond"] == "jacobi" else 0
        d.op_type = 1 if sv["operator"] == "fem" else 0
        d.lin_tol, d.lin_maxit, d.krylov = sv["tol"], sv["maxit"], sv["krylov"]
        if sv["newton"]:
            d.nonlinear = 1
            d.nl_abs, d.nl_rel, d.nl_maxit = sv["newton"]
        if sv["transient"]:
            d.transient = 1
            d.t0, d.tf, d.dt = sv["transient"]
        self.nsd = nsd
        self.h = L.refp_create(C.byref(d))
        if not self.h:
            raise ValueError(L.refp_last_error().decode())
        self.n = L.refp_num_free(self.h)
        self.nnodes = L.refp_num_nodes(self.h)

    def __del__(self):
        try:
            _refp_lib().refp_destroy(self.h)
        except Exception:
            pass

    def mesh(self, nelem, nfaces):
        xyz = np.zeros(self.nnodes * self.nsd)
        rng = np.zeros(nelem * nfaces, np.int32)
        _refp_lib().refp_mesh(self.h, _ptr(xyz), _ptr(rng))
        return xyz, rng

    def dofmap(self):
        t2a = np.zeros(self.nnodes, np.int32)
        _refp_lib().refp_dofmap(self.h, _ptr(t2a))
        return t2a

    def run(self):
        """The configured solve from the configured initial condition: (U over the free DOFs, converged)."""
        U = np.zeros(self.n)
        rc = _refp_lib().refp_run(self.h, _ptr(U))
        if rc < 0:
            raise RuntimeError(_refp_lib().refp_last_error().decode())
        return U, rc == 0

    def pattern(self):
        L = _refp_lib()
        nnz = L.refp_nnz(self.h)
        rp = np.zeros(self.n + 1, np.int64)
        col = np.zeros(max(nnz, 1), np.int64)
        L.refp_pattern(self.h, _ptr(rp), _ptr(col))
        return rp, col[:nnz]

    def assemble_matrix(self, formset, c=0.0, t=0.0, U=None, Udot=None):
        """formset 0 K; 1 K + c M; 2 K + K_T; 3 K + K_T + c M + M_T, with the problem's models."""
        L = _refp_lib()
        val = np.zeros(max(L.refp_nnz(self.h), 1))
        if L.refp_assemble_matrix(self.h, formset, c, t, _ptr(_f64(U)), _ptr(_f64(Udot)), _ptr(val)):
            raise RuntimeError(L.refp_last_error().decode())
        return val[:L.refp_nnz(self.h)]

    def assemble_vector(self, which, t=0.0, U=None, Udot=None):
        """which 0: load + natural BCs at t; 1: stiffness residual K(U) U (Full gather); 2: mass forms on Udot."""
        L = _refp_lib()
        out = np.zeros(self.n)
        if L.refp_assemble_vector(self.h, which, t, _ptr(_f64(U)), _ptr(_f64(Udot)), _ptr(out)):
            raise RuntimeError(L.refp_last_error().decode())
        return out


def ref_transient_adjoint(nel, theta, U0, dt, nsteps, Uobs, bc_val=None, tol=1e-14):
    """FP64 CPU discrete adjoint of `nsteps` Backward-Euler steps on the reference's own templates:
    3D Q1 block mesh, k_e = exp(theta_e), f = 1, Dirichlet constants `bc_val` (default 0) on every face,
    J = 0.5 ||U_N - Uobs||^2.  Forward steps by the reference's BackwardEulerStage; adjoint solves by its
    cg::Solver + Jacobi on its assembled K + M/dt; element terms by its DiffusionForm
    (ref_adjoint_gradient).  Returns (U_N, J, dJ/dtheta, the reference's CG iterations)."""
    bcs = {t: 0.0 for t in range(6)}
    bcs.update(bc_val or {})
    r = Reference(3, 1, 2, nel, [0, 0, 0], [1, 1, 1], list(range(6)), bc_kind=0, bc_val=bcs, src_kind=0, src_c=1.0,
                  k_elem=np.exp(theta))
    states = [np.array(U0, dtype=np.float64)]
    for _ in range(nsteps):
        U, _, rc = r.backward_euler(dt, 1, states[-1], tol=tol, maxit=100000)
        if rc:
            raise RuntimeError("reference step did not converge")
        states.append(U)
    rp, col = r.pattern()
    A = r.assemble_matrix("K+cM", 1.0 / dt)
    mu_next = np.zeros(r.n)
    g = np.zeros(len(theta))
    its = 0
    for k in range(nsteps, 0, -1):
        b = states[-1] - Uobs if k == nsteps else r.assemble_vector(3, Udot=mu_next) / dt
        mu, rep = ref_csr_solve(rp, col, A, b, x0=mu_next, tol=tol, maxit=100000)
        its += int(rep["iterations"])
        g += r.adjoint_gradient(states[k], mu)
        mu_next = mu
    J = 0.5 * float(np.sum((states[-1] - Uobs) ** 2))
    return states[-1], J, -np.exp(theta) * g, its


def ref_write_pmsh(path, nsd, order, nel, lo, hi, tag_map=None):
    """The reference's BlockMesh2D/3D mesh (boundary tags renumbered by tag_map) written by its own
    MeshIO::writeBinary to `path`; returns the mesh arrays (xyz, ien, rng) the reference built."""
    L = _refp_lib()
    d = _RefpDesc()
    d.nsd, d.order = nsd, order
    nel = list(nel) + [1] * (3 - len(nel))
    for i in range(3):
        d.nel[i] = nel[i]
    for i in range(nsd):
        d.lo[i], d.hi[i] = lo[i], hi[i]
    for t in range(6):
        d.tag_map[t] = (tag_map or {}).get(t, -1)
    if L.refp_write_pmsh(C.byref(d), path.encode()):
        raise RuntimeError(L.refp_last_error().decode())
