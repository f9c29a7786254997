"""Device-resident implicit cpGIMP engine (one problem instance, one GPU).

The Engine owns every device buffer (torch tensors used as plain CUDA memory)
and sequences one load step through the C ABI of libgeowarp_b200.so:

    reset -> [user BCs] -> cell sort -> P2G activation (+ pressure BCs)
          -> [u-p: consistent-mass projection, CG on the GPU]
          -> row compaction -> block-CSR pattern (once per step)
          -> Newton { residual + element tangent, ||R||, Krylov, u += delta }
          -> G2P + lp update

which is the order of advance_one_step in solvers/quasi_static_solver_2d.py:239-258,
solvers/quasi_static_coupled_solver_2d.py:274-313 and
solvers/quasi_static_coupled_solver_3d.py:258-420.  There is no CPU path: every
numerical step is a CUDA kernel of the library.
"""
import ctypes as C
import math

import numpy as np
import torch

from . import _lib as L

MODEL_IDS = {
    "Hencky elasticity": L.MODEL_HENCKY,
    "J2": L.MODEL_J2,
    "Neo-Hookean": L.MODEL_NEOHOOKEAN,
    "Linear elasticity": L.MODEL_LINEAR,
    "Drucker-Prager": L.MODEL_DP,
    "NorSand": L.MODEL_NORSAND,
}

PRECISIONS = {"fp64": L.PREC_F64, "mixed": L.PREC_F32}
# u-p mobility: constant k0, or the J-dependent law of Uzuoka & Borja (2012) Eq. 86
MOBILITY_LAWS = {"constant": 0, "Uzuoka-Borja": 1}
PRECONDS = {"diag": L.PRECOND_DIAG, "block": L.PRECOND_BLOCK, "mg": "mg"}
# Models whose load steps always start from zero, even with predict_increment:
# non-associated Drucker-Prager and softening NorSand, whose incremental problem
# can lose uniqueness.  There another starting iterate may converge to another
# branch than the zero start of the FP64 drop-in.
_NO_PREDICT_MODELS = (L.MODEL_DP, L.MODEL_NORSAND)


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def material_struct(mat):
    """gw_material_t from a reference-style material dict."""
    m = L.Material()
    name = mat["material_name"]
    if name not in MODEL_IDS:
        raise ValueError(f"Unimplemented material model: {name}")
    m.model = MODEL_IDS[name]
    m.youngs_modulus = float(mat.get("youngs_modulus", 0.0))
    m.poisson_ratio = float(mat.get("poisson_ratio", 0.0))
    m.kappa = float(mat.get("kappa", 0.0))
    m.friction_angle = float(mat.get("friction_angle", 0.0))
    m.dilation_angle = float(mat.get("dilation_angle", 0.0))
    m.cohesion = float(mat.get("cohesion", 0.0))
    m.shape_factor = float(mat.get("shape_factor", 0.0))
    m.dp_tension_cutoff = 1 if mat.get("tension_cutoff", True) else 0
    m.dp_tip_tangent = float(mat.get("tip_tangent_fraction", 0.0))
    m.ns_kappa = float(mat.get("kappa", 0.0)) if name == "NorSand" else 0.0
    for key, attr in (("tilde_lambda", "ns_tilde_lambda"), ("M", "ns_M"), ("N", "ns_N"), ("beta", "ns_beta"),
                      ("vc0", "ns_vc0"), ("p0", "ns_p0"), ("v0", "ns_v0"), ("h", "ns_h"),
                      ("shear_modulus", "ns_shear_modulus"), ("initial_volumetric_strain", "ns_eps_v0")):
        setattr(m, attr, float(mat.get(key, 0.0)))
    if name == "NorSand" and m.ns_beta == 0.0:
        m.ns_beta = 1.0
    return m


class _Buf:
    """Grow-only device byte buffer."""

    def __init__(self, device):
        self.device = device
        self.t = torch.empty(0, dtype=torch.uint8, device=device)

    def get(self, nbytes):
        nbytes = max(int(nbytes), 256)
        if self.t.numel() < nbytes:
            self.t = torch.empty(int(nbytes * 1.25) + 256, dtype=torch.uint8, device=self.device)
        return self.t


class Engine:
    """State and step sequencing for one problem.

    kind: 'solid2d' | 'coupled2d' | 'coupled3d'
    n_grid: cells per axis; h: cell sizes used by the shape functions (2D
    reference solvers use dx on both axes); h_nodes: cell sizes for nodal
    positions; domain_min/max: lp clipping box.
    """

    KINDS = {"solid2d": L.KIND_SOLID2D, "coupled2d": L.KIND_COUPLED2D, "coupled3d": L.KIND_COUPLED3D}

    def __init__(self, kind, n_grid, h, h_nodes, domain_min, domain_max, x_init, device=None,
                 precision="fp64", precond="mg", krylov_rtol=None, krylov_max_iter=20000, krylov="gmres",
                 restart=None):
        if not torch.cuda.is_available():
            raise RuntimeError("geowarp_b200 needs a CUDA device (there is no CPU fallback)")
        L.load()
        self.kind_name = kind
        self.kind = self.KINDS[kind]
        self.D = 2 if kind != "coupled3d" else 3
        self.nf = {"solid2d": 2, "coupled2d": 3, "coupled3d": 4}[kind]
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.n_grid = tuple(int(v) for v in n_grid)
        self.n_nodes = int(np.prod([v + 1 for v in self.n_grid]))
        self.n_cells = int(np.prod(self.n_grid))
        self.h = tuple(float(v) for v in h)
        self.h_nodes = tuple(float(v) for v in h_nodes)
        self.domain_min = tuple(float(v) for v in domain_min)
        self.domain_max = tuple(float(v) for v in domain_max)
        self.precision = precision
        self.prec = PRECISIONS[precision]
        self.precond = PRECONDS[precond]
        self.krylov_rtol = krylov_rtol if krylov_rtol is not None else (1e-12 if precision == "fp64" else 1e-6)
        self.final_krylov_rtol = 1e-6  # solve tolerance of the update taken at ||R|| < tol
        # inexact-Newton forcing (mixed precision only): each correction is
        # solved to rtol = clamp(forcing * tol / ||R||, krylov_rtol, forcing_max),
        # i.e. only as accurately as reaching ||R|| < tol needs; None keeps the
        # reference's full solves (the FP64 drop-in)
        self.newton_forcing = 0.1 if precision == "mixed" else None
        self.forcing_max = 0.1
        # lower bound of the adjoint's transpose-solve tolerance: in mixed
        # precision the FP32 transposed Jacobian fixes lambda to about 1e-5
        # relative (the gradient's distance to the FP64 one), so a tighter solve
        # changes nothing that the FP32 operator resolves
        self.adjoint_rtol_floor = 1e-5 if precision == "mixed" else 0.0
        # chord final update (mixed precision only): when the residual norms so
        # far predict ||R|| < tol at the next iterate, that iterate is checked
        # with a residual-only assembly first; if it has converged, the last
        # update (solved only to forcing_max) reuses the previous Jacobian
        # instead of assembling a new tangent
        self.final_chord = precision == "mixed"
        # Newton's starting iterate (mixed precision, 2D solid only): the previous
        # load step's converged increment on the new step's free DOFs, when the
        # previous step was current_step - 1 and its Newton loop reached
        # ||R|| < tol (gw_predict_increment).  Along a
        # load ramp consecutive increments differ by the change of the response,
        # so the first residual starts far below the zero iterate's.  The
        # converged state does not depend on the start; the reference (and the
        # FP64 drop-in) starts every load step from zero.  Not for the models of
        # _NO_PREDICT_MODELS.
        self.predict_increment = precision == "mixed" and kind == "solid2d"
        self._u_prev = None  # converged increment of load step _u_prev_step (node-indexed)
        self._u_prev_step = None
        self.krylov_max_iter = krylov_max_iter
        if krylov not in ("gmres", "bicgstab"):
            raise ValueError(f"unknown Krylov method {krylov!r}")
        self.krylov_method = krylov
        # flexible GMRES with a V-cycle needs few iterations; the Jacobi-preconditioned
        # one needs a long basis
        self.restart = int(restart) if restart is not None else (30 if precond == "mg" else 100)
        self.mw = 1 if self.D == 2 else 4

        dev = self.device
        f64 = dict(dtype=torch.float64, device=dev)
        x = torch.as_tensor(np.asarray(x_init, dtype=np.float64)).to(dev)
        self.N = x.shape[0]
        N = self.N
        self.x = x.contiguous()
        self.x0 = x.clone()
        self.lp = torch.zeros((N, self.D), **f64)
        ident = torch.tensor([[1.0 + 1e-7, 0, 0], [0, 1.0 - 1e-6, 0], [0, 0, 1.0]], **f64)
        self.F_old = ident.expand(N, 3, 3).contiguous()
        self.F_new = self.F_old.clone()
        self.b_old = self.F_old.clone()
        self.b_new = self.F_old.clone()
        self.sigma = torch.zeros((N, 3, 3), **f64)
        self.pressure = torch.zeros(N, **f64)
        self.pi_old = torch.zeros(N, **f64)
        self.pi_new = torch.zeros(N, **f64)
        self.ext_flag = torch.zeros(N, dtype=torch.bool, device=dev)
        self.trac_flag = torch.zeros(N, dtype=torch.bool, device=dev)
        self.pbc_flag = torch.zeros(N, dtype=torch.bool, device=dev)
        self.E = None  # optional per-particle Young's modulus [N]

        nn = self.n_nodes
        self.boundary = torch.zeros(self.nf * nn, dtype=torch.bool, device=dev)
        self.node_active = torch.zeros(nn, dtype=torch.uint8, device=dev)
        self.cell_span = torch.zeros(self.n_cells, dtype=torch.int32, device=dev)
        self.free_mask = torch.zeros(nn, dtype=torch.uint8, device=dev)
        self.node2row = torch.zeros(nn, dtype=torch.int32, device=dev)
        self.row2node = torch.zeros(nn, dtype=torch.int32, device=dev)
        self.stencil = torch.zeros(nn * self.mw, dtype=torch.int32, device=dev)
        self.u_new = torch.zeros(nn * self.nf, **f64)
        self.u_old = torch.zeros(nn * self.nf, **f64)
        self.keys = torch.zeros(N, dtype=torch.int32, device=dev)
        self.perm = torch.zeros(N, dtype=torch.int32, device=dev)
        self.force = torch.zeros(1, **f64)
        self.norm_dev = torch.zeros(1, **f64)
        self._sort_ws = _Buf(dev)
        self._scan_ws = _Buf(dev)
        self._asm_ws = _Buf(dev)  # particle records of the cell-coloured assembly
        self.deterministic_assembly = True
        self._kry_ws = _Buf(dev)
        self._norm_ws = torch.zeros(16384, dtype=torch.uint8, device=dev)
        self._row_ptr = torch.zeros(1, dtype=torch.int32, device=dev)
        self._cols = torch.zeros(1, dtype=torch.int32, device=dev)
        self._vals = _Buf(dev)
        self._R = torch.zeros(1, **f64)
        self._delta = torch.zeros(1, **f64)
        self._mg_plan = None
        self._mg_numeric = None  # (role of the last numeric phase, its GMRES iterations)
        self._gm_hint = 0  # iterations of this engine's last multigrid GMRES solve
        self.mg_lag = True  # Newton solves of a load step share one multigrid numeric phase
        # consistent-mass system (u-p kinds)
        if self.nf > self.D:
            self.touched = torch.zeros(nn, dtype=torch.uint8, device=dev)
            self.m_node2row = torch.zeros(nn, dtype=torch.int32, device=dev)
            self.m_row2node = torch.zeros(nn, dtype=torch.int32, device=dev)
            self.m_stencil = torch.zeros(nn * self.mw, dtype=torch.int32, device=dev)
            self._m_row_ptr = torch.zeros(1, dtype=torch.int32, device=dev)
            self._m_cols = torch.zeros(1, dtype=torch.int32, device=dev)
            self._m_vals = torch.zeros(1, **f64)
            self._m_rhs = torch.zeros(1, **f64)
            self._m_x = torch.zeros(1, **f64)
        self.n_rows = 0
        self.nnzb = 0
        self.m_rows = 0
        self.m_nnzb = 0
        self.step_params = {}
        self.line_search_growth = None  # e.g. 2.0 enables the backtracking safeguard
        self.line_search_max = 6
        self.log = []  # per Newton iteration: (step, it, ||R||, krylov iters, relres, status)

    # ------------------------------------------------------------------ structs
    def grid_struct(self):
        g = L.Grid()
        g.dim = self.D
        g.kind = self.kind
        g.nf = self.nf
        for k in range(3):
            g.n_grid[k] = self.n_grid[k] if k < self.D else 0
            g.h[k] = self.h[k] if k < self.D else 1.0
            g.inv_h[k] = 1.0 / self.h[k] if k < self.D else 1.0
            g.h_nodes[k] = self.h_nodes[k] if k < self.D else 1.0
            g.domain_min[k] = self.domain_min[k] if k < self.D else 0.0
            g.domain_max[k] = self.domain_max[k] if k < self.D else 0.0
        g.n_nodes = self.n_nodes
        return g

    def particles_struct(self):
        p = L.Particles()
        p.n = self.N
        p.x, p.x0, p.lp = _p(self.x), _p(self.x0), _p(self.lp)
        p.F_old, p.F_new, p.b_old, p.b_new = _p(self.F_old), _p(self.F_new), _p(self.b_old), _p(self.b_new)
        p.sigma, p.pressure, p.pi_old, p.pi_new = _p(self.sigma), _p(self.pressure), _p(self.pi_old), _p(self.pi_new)
        p.ext_flag, p.trac_flag, p.pbc_flag = _p(self.ext_flag), _p(self.trac_flag), _p(self.pbc_flag)
        p.E = _p(self.E)
        return p

    def bsr_struct(self, mass=False):
        b = L.Bsr()
        if mass:
            b.n_rows, b.nf, b.nnzb, b.mask_words = self.m_rows, 1, self.m_nnzb, self.mw
            b.row_ptr, b.cols, b.row2node, b.node2row = (_p(self._m_row_ptr), _p(self._m_cols), _p(self.m_row2node),
                                                         _p(self.m_node2row))
            b.stencil, b.vals = _p(self.m_stencil), _p(self._m_vals)
        else:
            b.n_rows, b.nf, b.nnzb, b.mask_words = self.n_rows, self.nf, self.nnzb, self.mw
            b.row_ptr, b.cols, b.row2node, b.node2row = (_p(self._row_ptr), _p(self._cols), _p(self.row2node),
                                                         _p(self.node2row))
            b.stencil, b.vals = _p(self.stencil), _p(self._vals.t)
        return b

    @property
    def stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    # ------------------------------------------------------------------ step pieces
    def reset(self, clear_boundary):
        self.u_old.zero_()
        self.u_new.zero_()
        self.node_active.zero_()
        self.cell_span.zero_()
        if clear_boundary:
            self.boundary.zero_()

    def sort_and_activate(self):
        g, pt, s = self.grid_struct(), self.particles_struct(), self.stream
        ws = self._sort_ws.get(L.load().gw_sort_workspace_bytes(self.N))
        L.call("gw_cell_sort", C.byref(g), C.byref(pt), _p(self.keys), _p(self.perm), _p(ws), s)
        L.call("gw_p2g_activate", C.byref(g), C.byref(pt), _p(self.perm), _p(self.node_active), _p(self.cell_span),
               _p(self.boundary), s)

    def _scan_ws_for(self, n):
        return self._scan_ws.get(L.load().gw_scan_workspace_bytes(int(n) + 1))

    def build_system(self):
        """Row compaction and block-CSR pattern, once per load step."""
        self._mg_plan = None  # the multigrid plan follows the pattern
        self._mg_numeric = None
        g, s = self.grid_struct(), self.stream
        nr = C.c_int32(0)
        L.call("gw_compact_rows", C.byref(g), _p(self.node_active), _p(self.boundary), _p(self.node2row),
               _p(self.row2node), _p(self.free_mask), C.byref(nr), _p(self._scan_ws_for(self.n_nodes)), s)
        self.n_rows = nr.value
        if self._row_ptr.numel() < self.n_rows + 1:
            self._row_ptr = torch.zeros(int((self.n_rows + 1) * 1.25) + 8, dtype=torch.int32, device=self.device)
        nnzb = C.c_int32(0)
        L.call("gw_pattern_count", C.byref(g), _p(self.cell_span), _p(self.node2row), _p(self.row2node),
               self.n_rows, _p(self.stencil), _p(self._row_ptr), C.byref(nnzb),
               _p(self._scan_ws_for(self.n_rows + 1)), s)
        self.nnzb = nnzb.value
        if self._cols.numel() < self.nnzb:
            self._cols = torch.zeros(int(self.nnzb * 1.25) + 8, dtype=torch.int32, device=self.device)
        vbytes = (8 if self.prec == L.PREC_F64 else 4) * self.nnzb * self.nf * self.nf
        self._vals.get(vbytes)
        b = self.bsr_struct()
        L.call("gw_pattern_fill", C.byref(g), C.byref(b), _p(self._cols), s)
        n = self.n_rows * self.nf
        if self._R.numel() < n:
            self._R = torch.zeros(int(n * 1.25) + 8, dtype=torch.float64, device=self.device)
            self._delta = torch.zeros_like(self._R)

    def project_pressure(self, cg_rtol=1e-13, lumped=False):
        """Projection of particle pressure to the nodes: consistent mass (GPU
        CG), or lumped (nodal pressure = sum N m p / sum N m)."""
        g, pt, s = self.grid_struct(), self.particles_struct(), self.stream
        self.touched.zero_()
        L.call("gw_touched_nodes", C.byref(g), _p(self.cell_span), _p(self.touched), s)
        nr = C.c_int32(0)
        L.call("gw_compact_rows", C.byref(g), _p(self.touched), _p(self.boundary), _p(self.m_node2row),
               _p(self.m_row2node), C.c_void_p(0), C.byref(nr), _p(self._scan_ws_for(self.n_nodes)), s)
        self.m_rows = nr.value
        if self._m_row_ptr.numel() < self.m_rows + 1:
            self._m_row_ptr = torch.zeros(int((self.m_rows + 1) * 1.25) + 8, dtype=torch.int32, device=self.device)
        nnzb = C.c_int32(0)
        L.call("gw_pattern_count", C.byref(g), _p(self.cell_span), _p(self.m_node2row), _p(self.m_row2node),
               self.m_rows, _p(self.m_stencil), _p(self._m_row_ptr), C.byref(nnzb),
               _p(self._scan_ws_for(self.m_rows + 1)), s)
        self.m_nnzb = nnzb.value
        if self._m_cols.numel() < self.m_nnzb:
            self._m_cols = torch.zeros(int(self.m_nnzb * 1.25) + 8, dtype=torch.int32, device=self.device)
            self._m_vals = torch.zeros(int(self.m_nnzb * 1.25) + 8, dtype=torch.float64, device=self.device)
        if self._m_rhs.numel() < self.m_rows:
            self._m_rhs = torch.zeros(int(self.m_rows * 1.25) + 8, dtype=torch.float64, device=self.device)
            self._m_x = torch.zeros_like(self._m_rhs)
        M = self.bsr_struct(mass=True)
        L.call("gw_pattern_fill", C.byref(g), C.byref(M), _p(self._m_cols), s)
        st = self.step_struct(0, 1)
        L.call("gw_mass_assemble", C.byref(g), C.byref(pt), _p(self.perm), C.byref(st), C.byref(M), _p(self._m_rhs), s)
        self._m_x.zero_()
        if lumped:
            L.call("gw_mass_lumped_solve", C.byref(M), _p(self._m_rhs), _p(self._m_x), s)
            self.mass_cg_iters = 0
        else:
            ws = self._kry_ws.get(L.load().gw_krylov_workspace_bytes(self.m_rows, 1, L.PREC_F64))
            it, rr = C.c_int32(0), C.c_double(0.0)
            rc = L.load().gw_bsr_krylov_solve(C.byref(M), L.PREC_F64, L.KRYLOV_CG, L.PRECOND_DIAG, _p(self._m_rhs),
                                              _p(self._m_x), cg_rtol, 100000, _p(ws), C.byref(it), C.byref(rr), s)
            if rc not in (L.GW_OK, L.GW_ENOCONV):
                L.check(rc, "consistent-mass CG")
            self.mass_cg_iters = it.value
        L.call("gw_set_nodal_pressure", C.byref(g), _p(self.m_row2node), self.m_rows, _p(self._m_x), _p(self.boundary),
               _p(self.node_active), _p(self.u_old), _p(self.u_new), s)

    def step_struct(self, current_step, total_steps):
        sp = self.step_params
        st = L.Step()
        st.current_step = float(current_step)
        st.total_steps = float(total_steps)
        st.gravity_mag = float(sp.get("gravity_mag", 0.0))
        st.gravity_full = 0 if sp.get("gravity_ramp", True) else 1
        st.mobility_law = MOBILITY_LAWS[sp.get("mobility_law", "constant")]
        for k in range(3):
            st.point_load[k] = float(sp.get("point_load", (0.0, 0.0, 0.0))[k])
            st.traction[k] = float(sp.get("traction", (0.0, 0.0, 0.0))[k])
        st.p_vol = float(sp["p_vol"])
        st.p_rho = float(sp["p_rho"])
        st.PPD = float(sp["PPD"])
        st.dt = float(sp.get("dt", 0.0))
        st.phi_initial = float(sp.get("phi_initial", 0.0))
        st.mobility = float(sp.get("mobility", 0.0))
        st.lp0 = float(sp["lp0"])
        fo = sp.get("footing")
        if fo is not None:
            st.has_footing = 1
            st.footing_min[0], st.footing_min[1] = fo["min"][0], fo["min"][1] if len(fo["min"]) > 1 else 0.0
            st.footing_max[0], st.footing_max[1] = fo["max"][0], fo["max"][1] if len(fo["max"]) > 1 else 0.0
            st.footing_initial_height = fo["initial_height"]
            st.footing_incr_disp = fo["incr_disp"]
            st.penalty_factor = fo["penalty_factor"]
            st.footing_stable = 1 if fo.get("stable", False) else 0
        return st

    def assemble(self, mat_struct, current_step, total_steps, want_K=True):
        """Residual and (want_K) element tangent: the deterministic cell-coloured
        assembly for the 2D kinds, the atomic one for 3D (or when
        deterministic_assembly is False)."""
        g, pt, s = self.grid_struct(), self.particles_struct(), self.stream
        st = self.step_struct(current_step, total_steps)
        A = self.bsr_struct()
        if not want_K:
            A.vals = None  # residual only: the row map is still required
        self.force.zero_()
        if self.D == 2 and self.deterministic_assembly:
            ws = self._asm_ws.get(L.load().gw_assemble_workspace_bytes(C.byref(g), self.N, self.prec))
            L.call("gw_assemble_sorted", C.byref(g), C.byref(mat_struct), C.byref(st), C.byref(pt), _p(self.perm),
                   _p(self.keys), _p(self.free_mask), _p(self.u_new), _p(self.u_old), C.byref(A), self.prec,
                   _p(self._R), _p(self.force), _p(ws), ws.numel(), s)
            return
        L.call("gw_assemble", C.byref(g), C.byref(mat_struct), C.byref(st), C.byref(pt), _p(self.perm),
               _p(self.free_mask), _p(self.u_new), _p(self.u_old), C.byref(A), self.prec, _p(self._R),
               _p(self.force), s)

    def residual_norm_async(self):
        n = self.n_rows * self.nf
        L.call("gw_norm2", _p(self._R), n, _p(self.norm_dev), _p(self._norm_ws), self.stream)

    def krylov(self, rtol=None):
        A = self.bsr_struct()
        n = self.n_rows * self.nf
        self._delta[:n].zero_()
        lib = L.load()
        it, rr = C.c_int32(0), C.c_double(0.0)
        rtol = rtol if rtol is not None else self.krylov_rtol
        if self.krylov_method == "gmres":
            return self.gmres_solve(A, self._R, self._delta, rtol, newton=True)
        if self.precond == "mg":
            raise ValueError("the multigrid preconditioner runs inside GMRES (krylov='gmres')")
        else:
            ws = self._kry_ws.get(lib.gw_krylov_workspace_bytes(self.n_rows, self.nf, self.prec))
            rc = lib.gw_bsr_krylov_solve(C.byref(A), self.prec, L.KRYLOV_BICGSTAB, self.precond, _p(self._R),
                                         _p(self._delta), rtol, self.krylov_max_iter, _p(ws), C.byref(it),
                                         C.byref(rr), self.stream)
        if rc not in (L.GW_OK, L.GW_ENOCONV, L.GW_EBREAKDOWN):
            L.check(rc, "Krylov")
        return it.value, rr.value, rc

    def gmres_solve(self, A, b, x, rtol, newton=False):
        """GMRES on block-CSR A (rows of this engine's active set): node-block /
        diagonal Jacobi (gw_bsr_gmres_solve) or a geometric-multigrid V-cycle
        on the background grid (gw_bsr_gmres_mg_solve).

        Multigrid: the coarse patterns are built once per load step.  With
        mg_lag set, a Newton solve that follows another Newton solve of the
        same load step reuses that solve's coarse operators and smoothers
        (plan.lag); GMRES still applies the current Jacobian, so only the
        preconditioner lags.  Any other solve (the adjoint's transpose), or a
        lagged solve that needed more than twice the iterations of the last
        fresh one plus five, makes the next solve rebuild them."""
        lib = L.load()
        it, rr = C.c_int32(0), C.c_double(0.0)
        if self.precond == "mg":
            g = self.grid_struct()
            nbytes = lib.gw_gmres_mg_workspace_bytes(C.byref(g), self.n_rows, self.nf, self.restart)
            ws = self._kry_ws.get(nbytes)
            plan = self._mg_plan
            if plan is None or plan.workspace != ws.data_ptr() or plan.fine_nnzb != A.nnzb:
                # coarse patterns: once per load step (the pattern is fixed within it)
                plan = L.MgPlan()
                L.call("gw_mg_plan_build", C.byref(g), C.byref(A), _p(ws), ws.numel(), C.byref(plan), self.stream)
                plan.last_iters = self._gm_hint  # first Arnoldi chunk: this engine's previous solve
                self._mg_plan = plan
                self._mg_numeric = None
            plan.lag = int(bool(self.mg_lag and newton and self._mg_numeric is not None
                                and self._mg_numeric[0] == "newton"))
            rc = lib.gw_bsr_gmres_mg_solve(C.byref(g), C.byref(A), self.prec, C.byref(plan), _p(b), _p(x), rtol,
                                           self.krylov_max_iter, self.restart, _p(ws), ws.numel(), C.byref(it),
                                           C.byref(rr), self.stream)
            self._gm_hint = plan.last_iters
            if not newton:
                self._mg_numeric = ("other", it.value)
            elif not plan.lag:
                self._mg_numeric = ("newton", it.value)
            elif it.value > 2 * self._mg_numeric[1] + 5:
                self._mg_numeric = None
        else:
            ws = self._kry_ws.get(lib.gw_gmres_workspace_bytes(self.n_rows, self.nf, self.restart))
            rc = lib.gw_bsr_gmres_solve(C.byref(A), self.prec, self.precond, _p(b), _p(x), rtol,
                                        self.krylov_max_iter, self.restart, _p(ws), C.byref(it), C.byref(rr),
                                        self.stream)
        if rc not in (L.GW_OK, L.GW_ENOCONV, L.GW_EBREAKDOWN):
            L.check(rc, "GMRES")
        return it.value, rr.value, rc

    def apply_increment(self):
        A = self.bsr_struct()
        L.call("gw_apply_increment", C.byref(A), _p(self._delta), _p(self.u_new), self.stream)

    def g2p(self, current_step, total_steps):
        g, pt = self.grid_struct(), self.particles_struct()
        st = self.step_struct(current_step, total_steps)
        L.call("gw_g2p", C.byref(g), C.byref(st), C.byref(pt), _p(self.u_new), _p(self.u_old), self.stream)

    def device_status(self):
        v = C.c_int32(0)
        L.call("gw_read_device_status", C.byref(v), self.stream)
        return v.value

    # ------------------------------------------------------------------ Newton
    def newton_rtol(self, nrm, tol):
        """Krylov tolerance of the Newton correction at residual norm nrm.

        Without forcing: krylov_rtol (None), or final_krylov_rtol for the last
        update, taken at ||R|| < tol.  With forcing f (mixed precision): the
        inexact-Newton bound f * tol / ||R||, clamped to [krylov_rtol,
        forcing_max]: the next residual is about rtol * ||R|| plus the
        quadratic and FP32-Jacobian terms, so f = 0.1 leaves it a decade under
        tol without solving the correction past what the tolerance needs."""
        if self.newton_forcing is None:
            return None if nrm >= tol else max(self.krylov_rtol, self.final_krylov_rtol)
        eta = self.newton_forcing * tol / nrm if nrm > 0 else self.forcing_max
        return min(self.forcing_max, max(self.krylov_rtol, eta))

    def newton(self, mat_struct, current_step, total_steps, n_iter, tol):
        """Newton loop with the reference's stopping rule
        (solvers/quasi_static_solver_2d.py:151-231): R is assembled before the
        update, the update is applied, then ||R|| < tol stops the loop.

        With line_search_growth set (extension, off by default), an iterate
        whose residual norm exceeds growth x the previous one is rejected and
        the previous Newton step is halved (at most line_search_max times per
        load step); accepted iterates follow the reference exactly.

        With final_chord (mixed precision), the last update -- taken at
        ||R|| < tol -- may use the previous iterate's Jacobian; with
        predict_increment the loop starts from the previous load step's
        converged increment instead of zero: see Engine.__init__."""
        its = 0
        predict = self.predict_increment and mat_struct.model not in _NO_PREDICT_MODELS
        if predict and self._u_prev is not None and self._u_prev_step == current_step - 1:
            L.call("gw_predict_increment", C.byref(self.bsr_struct()), _p(self.free_mask), _p(self._u_prev),
                   _p(self.u_new), self.stream)
        growth = self.line_search_growth
        prev = None  # (u before the last step, delta, ||R|| at u)
        n_bt = 0
        alpha = 1.0
        n = self.n_rows * self.nf
        norms = []  # ||R|| of the accepted iterates
        converged = False
        for it in range(n_iter):
            if (self.final_chord and not growth and len(norms) >= 2 and 0.0 < norms[-1] < norms[-2]
                    and norms[-1] * (norms[-1] / norms[-2]) < 0.5 * tol):
                self.assemble(mat_struct, current_step, total_steps, want_K=False)
                self.residual_norm_async()
                nrm = float(self.norm_dev.item())
                if nrm < tol:  # converged: the last update with the Jacobian already assembled
                    kit, relres, rc = self.krylov(self.newton_rtol(nrm, tol))
                    self.apply_increment()
                    its += 1
                    self.log.append((current_step, it, nrm, kit, relres, rc))
                    converged = True
                    break
            self.assemble(mat_struct, current_step, total_steps, want_K=True)
            self.residual_norm_async()
            nrm = float(self.norm_dev.item())
            if growth:
                if prev is not None and (not math.isfinite(nrm) or nrm > growth * prev[2]) and n_bt < self.line_search_max:
                    alpha *= 0.5
                    n_bt += 1
                    self.u_new.copy_(prev[0])
                    self._delta[:n].copy_(prev[1]).mul_(alpha)
                    self.apply_increment()
                    self.log.append((current_step, it, nrm, 0, alpha, "backtrack"))
                    continue
            # ||R|| < tol already: this update is the last one (the reference
            # applies it, then stops); a 1e-6 relative solve moves u by far
            # less than the converged tolerance and spares a Krylov solve that
            # would chase a residual at the FP64 rounding floor
            kit, relres, rc = self.krylov(self.newton_rtol(nrm, tol))
            if growth:
                prev = (self.u_new.clone(), self._delta[:n].clone(), nrm)
                alpha = 1.0
            self.apply_increment()
            its += 1
            norms.append(nrm)
            self.log.append((current_step, it, nrm, kit, relres, rc))
            if not math.isfinite(nrm):
                hist = "; ".join(f"it {l[1]}: |R|={l[2]:.3e} krylov {l[3]} relres {l[4]:.2e} rc {l[5]}"
                                 for l in self.log[-its:])
                raise L.GeoWarpError(L.GW_ENAN, "newton", f"non-finite residual norm at step {current_step} "
                                     f"(device status {self.device_status()}; {hist})")
            if nrm < tol:
                converged = True
                break
        # only a converged increment predicts the next step's: an unconverged
        # one (Newton at its iteration cap) is no estimate of the solution
        self._u_prev_step = None
        if predict and converged:
            if self._u_prev is None or self._u_prev.numel() != self.u_new.numel():
                self._u_prev = torch.empty_like(self.u_new)
            self._u_prev.copy_(self.u_new)
            self._u_prev_step = current_step
        return its

    # ------------------------------------------------------------------ host views
    def rows_to_field_major(self, vec_rows):
        """Scatter an active-row vector to the reference's field-major layout."""
        out = torch.zeros(self.nf * self.n_nodes, dtype=torch.float64, device=self.device)
        nodes = self.row2node[: self.n_rows].long()
        v = vec_rows[: self.n_rows * self.nf].view(self.n_rows, self.nf)
        for f in range(self.nf):
            out[f * self.n_nodes + nodes] = v[:, f]
        return out

    def node_to_field_major(self, u):
        return u.view(self.n_nodes, self.nf).t().reshape(-1).contiguous()

    def matrix_coo(self):
        """Field-major COO triplets (rows, cols, vals) of the assembled K, for checks."""
        nf, nr = self.nf, self.n_rows
        rp = self._row_ptr[: nr + 1].long()
        cols = self._cols[: self.nnzb].long()
        counts = rp[1:] - rp[:-1]
        brow = torch.repeat_interleave(torch.arange(nr, device=self.device), counts)
        vt = torch.float64 if self.prec == L.PREC_F64 else torch.float32
        vals = self._vals.t[: self.nnzb * nf * nf * (8 if vt == torch.float64 else 4)].view(vt).view(self.nnzb, nf, nf)
        r2n = self.row2node[:nr].long()
        rows_o, cols_o, vals_o = [], [], []
        for f in range(nf):
            for gcol in range(nf):
                rows_o.append(f * self.n_nodes + r2n[brow])
                cols_o.append(gcol * self.n_nodes + r2n[cols])
                vals_o.append(vals[:, f, gcol].double())
        return torch.cat(rows_o), torch.cat(cols_o), torch.cat(vals_o)
