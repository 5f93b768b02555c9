"""Device models against fixtures from the reference's own HeatProblem (ConductivityModel with an
anisotropic k(T) tensor, SpecificHeatModel with cp(T), TangentMassForm, Dirichlet and flux tags outside
0..5), through the C ABI: DOF map bit-exact, assembled matrices and vectors and a steady solution at
1e-12 relative."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def block(rsd, nsd, nel, order, retag):
    from importlib import import_module
    bm = import_module("residuum_solver_b200.blockmesh")
    xyz, ien, rng = bm.block_mesh(nsd, nel, [0] * nsd, [1] * nsd, order)
    rng = rng.copy()
    for a, b in retag.items():
        rng[rng == a] = b
    return xyz, ien, rng


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


def test_anisotropic_kT_cpT_tangent_mass_and_tags(rsd, ctx):
    g = golden("models_aniso_kT_cpT_hex.npz")
    xyz, ien, rng = block(rsd, 3, [4, 3, 3], 1, {0: 9})
    h = rsd.Heat(ctx, rsd.Mesh(ctx, 3, 1, xyz, ien, rng), 2, k_expr="1 + 0.2*T", dk_expr="0.2", k_tensor=g["tensor"],
                 rho=2.0, cp_expr="1 + 0.3*T", dcp_expr="0.3", src_expr="1 + x*y",
                 dirichlet={9: "0", 1: "1 + x*y"}, flux={2: ("1 + y", "0.5", "0")})
    t2a, _ = h.dofmap()
    assert (t2a == g["t2a"]).all()
    rp, col = h.K.pattern()
    assert (rp == g["row_ptr"]).all() and (col == g["col"]).all()
    t = float(g["t"])
    h.set_time(t)
    U, Ud = ctx.to_device(g["U"]), ctx.to_device(g["Udot"])
    for key, c in (("K", (1.0, 0.0, 0.0, 0.0)), ("K_cM", (1.0, 50.0, 0.0, 0.0)), ("K_KT", (1.0, 0.0, 1.0, 0.0)),
                   ("J_BE", (1.0, 50.0, 1.0, 1.0))):
        h.assemble_matrix(*c, U=U, Udot=Ud)
        assert rel(h.K.values(), g[key]) <= 1e-12, key
    out = ctx.array(h.n)
    h.assemble_vector(0, out)
    h.apply_natural(out)
    assert rel(out.download(), g["F_natural"]) <= 1e-12
    h.assemble_vector(1, out, U=U)
    assert rel(out.download(), g["R_diff"]) <= 1e-12
    h.assemble_vector(3, out, U=U, Udot=Ud)   # rho cp(T(U)) Mass on Udot
    assert rel(out.download(), g["M_Udot"]) <= 1e-12
    # the matrix-free Jacobian product (Diffusion + TangentDiffusion + c Mass + TangentMass) inverts the
    # assembled Jacobian's SpMV
    v = ctx.to_device(np.cos(np.arange(h.n) * 0.3))
    h.assemble_matrix(1.0, 50.0, 1.0, 1.0, U=U, Udot=Ud)
    y1 = ctx.array(h.n)
    h.K.spmv(v, y1)
    b = ctx.to_device(y1.download())
    x = ctx.array(h.n).zero()
    rep = h.solve_fem_forms(b, x, c_tdiff=1.0, c_mass=50.0, c_tmass=1.0, U=U, Udot=Ud, type=rsd.GMRES, tol=1e-13,
                            max_iters=5000, krylov_dim=30)
    assert rep["converged"]
    assert rel(x.download(), v.download()) <= 1e-9


def test_constant_anisotropic_steady_q2_quad(rsd, ctx):
    g = golden("models_aniso_quad_q2.npz")
    xyz, ien, rng = block(rsd, 2, [6, 5], 2, {3: 7})
    h = rsd.Heat(ctx, rsd.Mesh(ctx, 2, 2, xyz, ien, rng), 3, k_const=1.0, k_tensor=g["tensor"], src_expr="2 - x",
                 dirichlet={0: "x*y", 7: "1"})
    t2a, _ = h.dofmap()
    assert (t2a == g["t2a"]).all()
    U = ctx.array(h.n).zero()
    for op in (rsd.OP_CSR, rsd.OP_FEM):
        U.zero()
        rep = h.steady(U, tol=1e-12, max_iters=5000, operator_type=op)
        assert rep["converged"]
        assert rel(U.download(), g["U"]) <= 1e-10, op


def test_adjoint_rejects_a_nonsymmetric_tensor(rsd, ctx):
    xyz, ien, rng = block(rsd, 3, [2, 2, 2], 1, {})
    h = rsd.Heat(ctx, rsd.Mesh(ctx, 3, 1, xyz, ien, rng), 2, k_tensor=[[1, 0.5, 0], [0, 1, 0], [0, 0, 1]], src_expr="1",
                 dirichlet={t: "0" for t in range(6)})
    theta, T = ctx.array(8).zero(), ctx.array(h.n).zero()
    with pytest.raises(rsd.RsdError):
        h.forward(theta, T, tol=1e-10)


def test_initial_condition_expression(rsd, ctx):
    xyz, ien, rng = block(rsd, 3, [3, 2, 2], 1, {})
    h = rsd.Heat(ctx, rsd.Mesh(ctx, 3, 1, xyz, ien, rng), 2, dirichlet={0: "0"})
    t2a, a2t = h.dofmap()
    U = ctx.array(h.n)
    h.eval_nodal("x*y + 2*z + t", U, t=0.5)
    X = xyz.reshape(-1, 3)[a2t]
    assert np.allclose(U.download(), X[:, 0] * X[:, 1] + 2 * X[:, 2] + 0.5, rtol=1e-15, atol=1e-15)


@pytest.mark.parametrize("name,nsd,order,nq,nel,hi,kw", [
    ("monitors_q2_hex_kT.npz", 3, 2, 3, [3, 3, 2], [2.0, 1.0, 0.5],
     dict(k_expr="1 + 0.5*T", dk_expr="0.5", src_expr="10", dirichlet={0: "0", 1: "1"})),
    ("monitors_q1_quad.npz", 2, 1, 2, [6, 5], [1.5, 0.75],
     dict(rho=1.5, cp=0.8, src_expr="2*x*y", dirichlet={t: "(1-x)*(1-y)" for t in range(4)})),
])
def test_heat_flux_monitors(rsd, ctx, name, nsd, order, nq, nel, hi, kw):
    """HeatFlux monitors (weak reaction and strong boundary quadrature, Integral and Average, steady
    and transient) against the reference's own monitor groups."""
    from importlib import import_module
    bm = import_module("residuum_solver_b200.blockmesh")
    g = golden(name)
    xyz, ien, rng = bm.block_mesh(nsd, nel, [0] * nsd, hi, order)
    h = rsd.Heat(ctx, rsd.Mesh(ctx, nsd, order, xyz, ien, rng), nq, **kw)
    U, Ud = ctx.to_device(g["U"]), ctx.to_device(g["Udot"])
    for method in ("weak", "strong"):
        for red in ("integral", "average"):
            v, m = h.boundary_flux(g["tags"], U, Ud, method=method, reduction=red)
            assert rel(v, g[f"{method}_{red}"]) <= 1e-12, (method, red)
            assert np.all(m > 0)
    for red in ("integral", "average"):
        v, _ = h.boundary_flux(g["tags"], U, Ud, method="weak", reduction=red, transient=True)
        assert rel(v, g[f"weak_transient_{red}"]) <= 1e-12, red


def test_pmsh_mesh_solves_like_the_block_mesh(rsd, ctx):
    """A PMSH file written by the reference's MeshIO (block tag 0 renumbered to 9) read into a device
    mesh gives the DOF map and steady solution of the same mesh built in memory."""
    import os
    from conftest import GOLDEN
    path = os.path.join(GOLDEN, "block_q2_hex_3x2x2.pmsh")
    g = golden("block_q2_hex_3x2x2.npz")
    bc = {9: "x*y", 1: "1"}
    hp = rsd.Heat(ctx, rsd.PmshMesh(ctx, path), 3, src_expr="1", dirichlet=bc)
    hb = rsd.Heat(ctx, rsd.Mesh(ctx, 3, 2, g["xyz"], g["ien"], g["rng"]), 3, src_expr="1", dirichlet=bc)
    assert (hp.dofmap()[0] == hb.dofmap()[0]).all()
    Up, Ub = ctx.array(hp.n).zero(), ctx.array(hb.n).zero()
    hp.steady(Up, tol=1e-12)
    hb.steady(Ub, tol=1e-12)
    # the element vectors sum by atomics, so the two solves agree to rounding, not bit for bit
    assert rel(Up.download(), Ub.download()) <= 1e-10


@pytest.mark.parametrize("nsd,order,nel,dirichlet,perm", [
    (3, 1, [7, 6, 5], {0: "0", 3: "x", 5: "1"}, False),
    (3, 2, [4, 3, 3], {9: "0", 1: "1"}, True),
    (2, 3, [6, 4], {0: "0", 2: "y", 3: "1"}, True),
    (2, 1, [9, 8], {}, False),
])
def test_device_setup_matches_host_setup(rsd, ctx, monkeypatch, nsd, order, nel, dirichlet, perm):
    """The DOF map and CSR pattern built on the device (the default) equal the host build
    (RSD_HOST_SETUP=1) bit for bit, on block meshes and on block meshes with shuffled node numbers; the
    steady solutions on either agree to rounding (element vectors sum by atomics)."""
    from importlib import import_module
    bm = import_module("residuum_solver_b200.blockmesh")
    xyz, ien, rng = bm.block_mesh(nsd, nel, [0] * nsd, [1] * nsd, order)
    rng = rng.copy()
    if 9 in dirichlet:
        rng[rng == 0] = 9
    if perm:
        nn = xyz.size // nsd
        p = np.random.default_rng(1).permutation(nn)      # new id of old node v is p[v]
        x2 = np.empty_like(xyz.reshape(nn, nsd))
        x2[p] = xyz.reshape(nn, nsd)
        xyz, ien = x2.reshape(-1), p[ien]
    out = []
    for host in ("1", "0"):
        monkeypatch.setenv("RSD_HOST_SETUP", host)
        h = rsd.Heat(ctx, rsd.Mesh(ctx, nsd, order, xyz, ien, rng), order + 1, src_expr="1", dirichlet=dirichlet)
        t2a, a2t = h.dofmap()
        rp, col = h.K.pattern()
        U = ctx.array(h.n).zero()
        if dirichlet:     # without an essential tag the steady problem is singular
            h.steady(U, tol=1e-12, max_iters=5000)
        out.append((t2a, a2t, rp, col, U.download()))
    for a, b in zip(out[0][:4], out[1][:4]):
        assert np.array_equal(a, b)
    if dirichlet:
        assert rel(out[0][4], out[1][4]) <= 1e-10
