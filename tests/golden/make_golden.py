"""Generate the golden fixtures in this folder from the reference's own templates.

    python tests/golden/make_golden.py [main] [adjoint] [fem] [models] [transient_adjoint] [monitors] [pmsh]

Every array comes from oracle/_ref/libresiduum_ref.so, i.e. the unmodified Residuum templates
(Assembler<CPU>, BoundaryApplicator<CPU>, TopologicalDOF, cg/gmres::Solver, SteadyStage,
BackwardEulerStage, NewtonRunner, and for the `models` group HeatProblem itself with its
ConductivityModel and SpecificHeatModel) compiled from the reference tree by oracle/Makefile.  The
fixtures are small so that the GPU tests can pin the CUDA path to the reference on a machine
without the reference tree.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
import oracle  # noqa: E402


def save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(path, {k: np.asarray(v).shape for k, v in arrays.items()})


def element_case(name, nsd, order, nq, nel, lo, hi, ess, bc_kind, src_kind, src_c, k_a=1.0, k_b=0.0, k_elem=None,
                 bc_val=None, seed=0):
    r = oracle.Reference(nsd, order, nq, nel, lo, hi, ess, bc_kind=bc_kind, bc_val=bc_val, src_kind=src_kind,
                         src_c=src_c, k_a=k_a, k_b=k_b, k_elem=k_elem)
    t2a, a2t = r.dofmap()
    rp, col = r.pattern()
    rng = np.random.default_rng(seed)
    U = 0.1 * rng.standard_normal(r.n)
    Ud = rng.standard_normal(r.n)
    ones = np.ones(r.n)
    F = r.assemble_vector(0)
    arrays = dict(t2a=t2a, a2t=a2t, row_ptr=rp, col=col, U=U, Udot=Ud,
                  K=r.assemble_matrix("K", U=U), K_cM=r.assemble_matrix("K+cM", 7.5, U=U),
                  K_KT=r.assemble_matrix("K+KT", U=U), F=F,
                  lift=r.lift(F, "K") - F, lift_cM=r.lift(F, "K+cM", 7.5) - F,
                  O_ones=r.assemble_vector(4, 0.0, operand=ones), O_cM=r.assemble_vector(4, 2.5, operand=Ud),
                  R_diff=r.assemble_vector(1, U=U), M_U=r.assemble_vector(2, U=U), M_Udot=r.assemble_vector(3, Udot=Ud),
                  diag=r.diagonal("K+cM", 7.5, U=U))
    if k_elem is not None:
        arrays["k_elem"] = np.asarray(k_elem)
    save(name, **arrays)
    return r


def main():
    # reference fem-tier fixtures: 4x4 Q1 on [0,4]^2, g = x on LEFT/RIGHT/TOP, f = x*y
    # (tests/integration/fem/heateq/cpu/HeatEquationMinimal2D.cpp) and 4^3 Q1 on [0,4]^3, g = x on the
    # four lateral faces, f = x*y*z (HeatEquationMinimal3D.cpp)
    element_case("q1_quad_4x4.npz", 2, 1, 2, [4, 4], [0, 0], [4, 4], [0, 1, 3], 1, 1, 1.0)
    element_case("q1_hex_4x4x4.npz", 3, 1, 2, [4, 4, 4], [0, 0, 0], [4, 4, 4], [0, 1, 2, 3], 1, 1, 1.0)
    # Q2 hex with k(T) = 1 + 0.5 T, Dirichlet 0 / 1 on x = 0 / 1 (the 48^3 Q2 nonlinear configuration's physics)
    element_case("q2_hex_3x3x2.npz", 3, 2, 3, [3, 3, 2], [0, 0, 0], [1, 1, 1], [0, 1], 0, 0, 10.0, k_a=1.0, k_b=0.5,
                 bc_val={0: 0.0, 1: 1.0})
    # Q2 quad with per-element conductivity and g = (1-x)(1-y)
    ke = np.exp(np.random.default_rng(7).standard_normal(15))
    element_case("q2_quad_kelem.npz", 2, 2, 3, [5, 3], [0, 0], [1, 1], [0, 1, 2, 3], 2, 0, 1.0, k_elem=ke)

    # steady 2D Q1 16x16, T = (1-x)(1-y) on all sides, CG + Jacobi to 1e-10 (the 64x64 configuration's physics)
    r = oracle.Reference(2, 1, 2, [16, 16], [0, 0], [1, 1], [0, 1, 2, 3], bc_kind=2)
    U, rep = r.steady(0, 1, 1e-10, 1000)
    save("steady_q1_quad_16.npz", U=U, iterations=rep["iterations"], finalResidual=rep["finalResidual"],
         initialResidual=rep["initialResidual"])
    U, rep = r.steady(1, 1, 1e-10, 1000, 7)
    save("steady_gmres7_q1_quad_16.npz", U=U, iterations=rep["iterations"], finalResidual=rep["finalResidual"])

    # Backward Euler, 3D Q1 6x5x4, Dirichlet 0, dt = 1e-2, 5 steps, CG + Jacobi 1e-8
    r = oracle.Reference(3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], list(range(6)), bc_kind=0)
    U0 = np.sin(np.arange(r.n) * 0.37)
    U, res, rc = r.backward_euler(1e-2, 5, U0, tol=1e-8)
    save("be_q1_hex_6x5x4.npz", U0=U0, U=U, residual=res)

    # Newton + GMRES(30) + Jacobi, Q2 hex 3^3, k = 1 + 0.5 T, f = 10, T = 0 / 1 on x = 0 / 1
    r = oracle.Reference(3, 2, 3, [3, 3, 3], [0, 0, 0], [1, 1, 1], [0, 1], bc_kind=0, bc_val={0: 0.0, 1: 1.0},
                         src_kind=0, src_c=10.0, k_a=1.0, k_b=0.5)
    U, rep = r.newton(1e-10, 1e-10, 50, 1, 1, 1e-12, 1000, 30)
    save("newton_q2_hex_3.npz", U=U, iterations=rep["iterations"], finalResidual=rep["finalResidual"])


def adjoint():
    # adjoint pair: 3D Q1 6x5x4 on the unit cube, k_e = exp(theta_e), f = 1, T = 0 on every face but
    # x = 1 (T = 0.5, so the gradient carries the lift's dependence on k); forward and adjoint solves
    # by the reference CG + Jacobi to 1e-14, the element gradient by the reference DiffusionForm
    rng = np.random.default_rng(55)
    theta = 0.5 * rng.standard_normal(6 * 5 * 4)
    r = oracle.Reference(3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], list(range(6)), bc_kind=0, bc_val={1: 0.5},
                         src_kind=0, src_c=1.0, k_elem=np.exp(theta))
    T, rep = r.steady(0, 1, 1e-14, 10000)
    Tobs = 0.05 * np.sin(1.7 * np.arange(r.n))
    rp, col = r.pattern()
    K = r.assemble_matrix("K")
    lam, lrep = oracle.ref_csr_solve(rp, col, K, T - Tobs, tol=1e-14, maxit=10000)
    g = r.adjoint_gradient(T, lam)
    grad = -np.exp(theta) * g
    # central differences of J through the reference forward solve, as a check of the generator
    d = rng.standard_normal(theta.size)
    d /= np.linalg.norm(d)
    h = 1e-6

    def J(th):
        rr = oracle.Reference(3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], list(range(6)), bc_kind=0, bc_val={1: 0.5},
                              src_kind=0, src_c=1.0, k_elem=np.exp(th))
        Tt, _ = rr.steady(0, 1, 1e-14, 10000)
        return 0.5 * np.sum((Tt - Tobs) ** 2)

    fd = (J(theta + h * d) - J(theta - h * d)) / (2 * h)
    assert abs(fd - grad @ d) <= 1e-6 * abs(fd), (fd, grad @ d)
    save("adjoint_q1_hex_6x5x4.npz", theta=theta, T=T, Tobs=Tobs, lam=lam, g=g, grad=grad, fd_dir=d, fd=fd)


def fem():
    # the matrix-free operator (LinearSolverConfig operator type "fem": FEMOperator, CG + Jacobi from
    # the element diagonal) through the reference's own stages
    r = oracle.Reference(3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], [0, 1, 2, 3], bc_kind=1, src_kind=1, src_c=1.0)
    r.set_operator("fem")
    U, rep = r.steady(0, 1, 1e-10, 1000)
    save("fem_steady_q1_hex_6x5x4.npz", U=U, iterations=rep["iterations"], initialResidual=rep["initialResidual"],
         finalResidual=rep["finalResidual"])
    r = oracle.Reference(3, 1, 2, [6, 5, 4], [0, 0, 0], [1, 1, 1], list(range(6)), bc_kind=0)
    r.set_operator("fem")
    U0 = np.sin(np.arange(r.n) * 0.37)
    U, res, rc, st = r.backward_euler(1e-2, 5, U0, tol=1e-8, stats=True)
    assert rc == 0
    save("fem_be_q1_hex_6x5x4.npz", U0=U0, U=U, residual=res, iterations=st[:, 2].astype(np.int64))
    ke = np.exp(np.random.default_rng(7).standard_normal(15))
    r = oracle.Reference(2, 2, 3, [5, 3], [0, 0], [1, 1], [0, 1, 2, 3], bc_kind=2, src_kind=0, src_c=1.0, k_elem=ke)
    r.set_operator("fem")
    U, rep = r.steady(0, 1, 1e-10, 1000)
    save("fem_steady_q2_quad_kelem.npz", k_elem=ke, U=U, iterations=rep["iterations"])
    r = oracle.Reference(3, 2, 3, [3, 3, 2], [0, 0, 0], [1, 1, 1], [0, 1], bc_kind=0, bc_val={0: 0.0, 1: 1.0},
                         src_kind=0, src_c=10.0)
    r.set_operator("fem")
    U, rep = r.steady(0, 1, 1e-10, 1000)
    save("fem_steady_q2_hex_3x3x2.npz", U=U, iterations=rep["iterations"])
    # GMRES(7) + Jacobi over the matrix-free operator, the 16x16 Q1 steady problem
    r = oracle.Reference(2, 1, 2, [16, 16], [0, 0], [1, 1], [0, 1, 2, 3], bc_kind=2)
    r.set_operator("fem")
    U, rep = r.steady(1, 1, 1e-10, 1000, 7)
    save("fem_steady_gmres7_q1_quad_16.npz", U=U, iterations=rep["iterations"], finalResidual=rep["finalResidual"])
    # Newton + GMRES(30) + Jacobi with the Jacobian forms applied matrix-free (the Newton fixture's problem)
    r = oracle.Reference(3, 2, 3, [3, 3, 3], [0, 0, 0], [1, 1, 1], [0, 1], bc_kind=0, bc_val={0: 0.0, 1: 1.0},
                         src_kind=0, src_c=10.0, k_a=1.0, k_b=0.5)
    r.set_operator("fem")
    U, rep = r.newton(1e-10, 1e-10, 50, 1, 1, 1e-12, 1000, 30)
    save("fem_newton_q2_hex_3.npz", U=U, iterations=rep["iterations"], finalResidual=rep["finalResidual"])
    # k(T) = 1 + 0.5 T in a linear stage: the operator's state is the solve's own iterate (the stage
    # binds its state to U, which the solver updates in place), so the operator changes as CG runs
    r = oracle.Reference(3, 2, 3, [3, 3, 2], [0, 0, 0], [1, 1, 1], [0, 1], bc_kind=0, bc_val={0: 0.0, 1: 1.0},
                         src_kind=0, src_c=10.0, k_a=1.0, k_b=0.5)
    r.set_operator("fem")
    U, rep = r.steady(0, 1, 1e-12, 1000)
    save("fem_steady_q2_hex_kT.npz", U=U, iterations=rep["iterations"], converged=rep["converged"])


# the conductivity tensor of the model fixtures: not symmetric, so that K = k kS and kS^T cannot be
# confused
ANISO_3D = [[2.0, 0.3, 0.0], [0.1, 1.0, 0.2], [0.0, 0.05, 0.5]]


def models():
    """Fixtures from the reference's own HeatProblem (oracle/ref_problem.cpp, its ConductivityModel and
    SpecificHeatModel): anisotropic k(T), cp(T) with TangentMass, a renumbered Dirichlet tag (block
    tag 0 -> 9), a flux boundary and an expression source; and a steady Q2 quad with a constant
    anisotropic tensor and a renumbered tag (3 -> 7)."""
    r = oracle.RefProblem(3, 1, 2, [4, 3, 3], [0, 0, 0], [1, 1, 1],
                          conductivity=("k(T) tensor", ANISO_3D, "1 + 0.2*T", "0.2"), rho=2.0,
                          specific_heat=("cp(T)", "1 + 0.3*T", "0.3"), source="1 + x*y",
                          bcs=[(9, "value", "0"), (1, "value", "1 + x*y"), (2, "flux", ["1 + y", "0.5", "0"])],
                          tag_map={0: 9}, solver=dict(type="gmres", tol=1e-12, newton=(1e-10, 1e-10, 30), transient=(0.0, 0.03, 0.01)))
    rng = np.random.default_rng(11)
    U = 0.3 * rng.standard_normal(r.n) + 0.5
    Ud = rng.standard_normal(r.n)
    rp, col = r.pattern()
    t = 0.3
    save("models_aniso_kT_cpT_hex.npz", t2a=r.dofmap(), row_ptr=rp, col=col, U=U, Udot=Ud, t=t, tensor=np.array(ANISO_3D),
         K=r.assemble_matrix(0, t=t, U=U, Udot=Ud), K_cM=r.assemble_matrix(1, 50.0, t=t, U=U, Udot=Ud),
         K_KT=r.assemble_matrix(2, t=t, U=U, Udot=Ud), J_BE=r.assemble_matrix(3, 50.0, t=t, U=U, Udot=Ud),
         F_natural=r.assemble_vector(0, t=t, U=U, Udot=Ud), R_diff=r.assemble_vector(1, t=t, U=U, Udot=Ud),
         M_Udot=r.assemble_vector(2, t=t, U=U, Udot=Ud))
    tensor2 = [[1.5, 0.4], [0.4, 0.8]]
    r = oracle.RefProblem(2, 2, 3, [6, 5], [0, 0], [1, 1], conductivity=("anisotropic", tensor2), source="2 - x",
                          bcs=[(0, "value", "x*y"), (7, "value", "1")], tag_map={3: 7}, solver=dict(tol=1e-12))
    Us, ok = r.run()
    assert ok
    save("models_aniso_quad_q2.npz", t2a=r.dofmap(), tensor=np.array(tensor2), U=Us)


def transient_adjoint():
    """Transient adjoint fixture: 3D Q1 6x5x4, k_e = exp(theta_e), f = 1, T = 0.5 on x = 1 and 0 on the
    other faces, 7 Backward-Euler steps of dt = 0.01 from U0, J = 0.5 ||U_7 - U_obs||^2; the FP64 CPU
    adjoint on the reference's templates (oracle.ref_transient_adjoint), checked here against central
    differences through the reference's own steps."""
    rng = np.random.default_rng(77)
    nel, dt, N = [6, 5, 4], 0.01, 7
    theta = 0.5 * rng.standard_normal(6 * 5 * 4)
    r = oracle.Reference(3, 1, 2, nel, [0, 0, 0], [1, 1, 1], list(range(6)), bc_kind=0, bc_val={1: 0.5})
    n = r.n
    U0 = 0.3 * np.sin(np.arange(n) * 0.41)
    Uobs = 0.05 * np.cos(np.arange(n) * 1.3)
    UN, J, grad, its = oracle.ref_transient_adjoint(nel, theta, U0, dt, N, Uobs, bc_val={1: 0.5})
    d = rng.standard_normal(theta.size)
    d /= np.linalg.norm(d)
    h = 1e-6
    Jp = oracle.ref_transient_adjoint(nel, theta + h * d, U0, dt, N, Uobs, bc_val={1: 0.5})[1]
    Jm = oracle.ref_transient_adjoint(nel, theta - h * d, U0, dt, N, Uobs, bc_val={1: 0.5})[1]
    fd = (Jp - Jm) / (2 * h)
    assert abs(fd - grad @ d) <= 1e-6 * abs(fd), (fd, grad @ d)
    save("transient_adjoint_q1_hex_6x5x4.npz", theta=theta, U0=U0, Uobs=Uobs, dt=dt, nsteps=N, UN=UN, J=J, grad=grad,
         fd_dir=d, fd=fd)


def monitors():
    """HeatFlux monitors through the reference's own monitor groups (oracle/ref_harness.cpp builds them
    as HeatProblem::makeMonitorGroup does): the weak (boundary reaction, steady and transient) and
    strong (boundary quadrature of HeatFluxIntegrand) methods, Integral and Average, on a Q2 hex box
    [0,2]x[0,1]x[0,0.5] with k(T) = 1 + 0.5 T and a 2D Q1 quad [0,1.5]x[0,0.75] with g = (1-x)(1-y)."""
    cases = {
        "monitors_q2_hex_kT.npz": dict(args=(3, 2, 3, [3, 3, 2], [0, 0, 0], [2.0, 1.0, 0.5], [0, 1]),
                                       kw=dict(bc_kind=0, bc_val={0: 0.0, 1: 1.0}, src_kind=0, src_c=10.0, k_a=1.0, k_b=0.5),
                                       tags=[0, 1, 2, 4]),
        "monitors_q1_quad.npz": dict(args=(2, 1, 2, [6, 5], [0, 0], [1.5, 0.75], [0, 1, 2, 3]),
                                     kw=dict(bc_kind=2, src_kind=1, src_c=2.0, rho=1.5, cp=0.8), tags=[0, 1, 2, 3]),
    }
    for name, c in cases.items():
        r = oracle.Reference(*c["args"], **c["kw"])
        rng = np.random.default_rng(5)
        U = 0.4 * rng.standard_normal(r.n) + 0.3
        Ud = rng.standard_normal(r.n)
        arrays = dict(tags=np.array(c["tags"], np.int32), U=U, Udot=Ud)
        for method in ("weak", "strong"):
            for red in ("integral", "average"):
                arrays[f"{method}_{red}"] = r.boundary_flux(c["tags"], U, Ud, method, red, False)
        for red in ("integral", "average"):
            arrays[f"weak_transient_{red}"] = r.boundary_flux(c["tags"], U, Ud, "weak", red, True)
        save(name, **arrays)


def pmsh():
    """PMSH mesh files written by the reference's own MeshIO::writeBinary from its block meshes (a Q2 hex
    box with tag 0 renumbered to 9, a Q1 quad), with the reference's arrays beside them."""
    for name, args, tags in (("block_q2_hex_3x2x2", (3, 2, [3, 2, 2], [0, 0, 0], [1.0, 0.5, 0.5]), {0: 9}),
                             ("block_q1_quad_5x4", (2, 1, [5, 4], [0, 0], [1.0, 1.0]), None)):
        path = os.path.join(HERE, name + ".pmsh")
        oracle.ref_write_pmsh(path, *args, tag_map=tags)
        print(path, os.path.getsize(path))
        nsd, order, nel, lo, hi = args
        m = oracle.BlockMesh(nsd, nel, lo, hi, order)
        rng = m.rng.copy()
        for a, b in (tags or {}).items():
            rng[rng == a] = b
        save(name + ".npz", xyz=m.xyz, ien=m.ien, rng=rng)


GROUPS = {"main": main, "adjoint": adjoint, "fem": fem, "models": models, "transient_adjoint": transient_adjoint,
          "monitors": monitors, "pmsh": pmsh}

if __name__ == "__main__":
    if not oracle.reference_available():
        sys.exit("oracle/_ref/libresiduum_ref.so is missing: run make -C oracle (needs the reference tree)")
    for name in sys.argv[1:] or list(GROUPS):
        GROUPS[name]()
