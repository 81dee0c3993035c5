"""Host-side mirror of BoSSS's operator registration and evaluator API.

The names and argument meanings follow the reference so that a test (or a C#
port of this file through P/Invoke) reads like the reference's own code:

* ``DifferentialOperator(DomainVarNames, ParameterVarNames, CodomainVarNames,
  QuadOrderFunc)`` -- ``DifferentialOperator.cs:452-490``;
  ``op.EquationComponents[cod].Add(component)``; ``op.Commit()`` (``:658-670``);
* ``op.GetEvaluatorEx(DomainFields, ParameterMap, CodomainVarMap)``
  (``:1013-1033``) returns an evaluator with
  ``Evaluate(alpha, beta, output)`` (``IEvaluator.cs:81-97``):
  ``output = beta*output + alpha*Op(DomainFields)``;
* equation components carry the reference class names (``ScalarTransportFlux``,
  ``SIPLaplace``, ``OptimizedHLLCDensityFlux``, ...).

Every evaluation runs through the C-ABI of ``libbosss_b200.so``; components
without a device functor fail at ``GetEvaluatorEx`` with
``BosssError(ERR_UNSUPPORTED_COMPONENT)`` -- there is no CPU fallback.
"""
import ctypes

import numpy as np

from . import _capi as C

# ----------------------------------------------------------------------------- quadrature orders


class QuadOrderFunc:
    """QuadOrderFunc.cs: each factory returns a (kind, parameter) descriptor."""

    @staticmethod
    def FixedOrder(order):
        return (C.QUAD_FIXED, int(order))

    @staticmethod
    def Linear():
        return (C.QUAD_LINEAR, 1)

    @staticmethod
    def NonLinear(NonLinDeg):
        return (C.QUAD_NONLINEAR, int(NonLinDeg))

    @staticmethod
    def MaxDegTimesTwo():
        return (C.QUAD_MAXDEG_TIMES_TWO, 0)

    @staticmethod
    def SumOfMaxDegrees(NonLinDeg=1, RoundUp=True):
        return (C.QUAD_SUM_OF_MAX_DEGREES if RoundUp else C.QUAD_NONLINEAR, int(NonLinDeg))


# ----------------------------------------------------------------------------- grids and fields


class CartesianGrid:
    """Uniform Cartesian grid as built by ``Grid2D.Cartesian2DGrid`` /
    ``Grid3D.Cartesian3DGrid`` from ``linspace`` node vectors. Local cell order is the
    generator's (x slowest, last axis fastest; ``Grid3D.cs:232-249``)."""

    def __init__(self, nodes, periodic, cell_order=C.CELLS_GENERATOR):
        self.dim = len(nodes)
        if self.dim not in (2, 3):
            raise ValueError("grid dimension must be 2 or 3")
        self.n, self.lo, self.hi = [], [], []
        for x in nodes:
            x = np.asarray(x, dtype=np.float64)
            if x.ndim != 1 or len(x) < 2:
                raise ValueError("node vectors need at least two entries")
            h = np.diff(x)
            if not np.allclose(h, h[0], rtol=1e-12, atol=0):
                raise ValueError("the device path supports uniform (linspace) node vectors only")
            self.n.append(len(x) - 1)
            self.lo.append(float(x[0]))
            self.hi.append(float(x[-1]))
        self.periodic = [bool(p) for p in periodic]
        self.cell_order = cell_order

    @property
    def NoOfCells(self):
        return int(np.prod(self.n))

    def desc(self):
        g = C.GridDesc()
        g.dim = self.dim
        for d in range(3):
            g.n[d] = self.n[d] if d < self.dim else 1
            g.lo[d] = self.lo[d] if d < self.dim else 0.0
            g.hi[d] = self.hi[d] if d < self.dim else 1.0
            g.periodic[d] = int(self.periodic[d]) if d < self.dim else 0
        g.cell_order = self.cell_order
        return g

    def cell_ijk(self):
        """(J, dim) integer cell indices in local order."""
        J = self.NoOfCells
        j = np.arange(J)
        if self.cell_order == C.CELLS_GENERATOR or self.dim == 2:
            # generator order; in 2D also the GlobalID order (Grid2D.cs:182)
            idx = np.unravel_index(j, self.n)                 # x slowest
        else:
            idx = np.unravel_index(j, self.n[::-1])[::-1]     # x fastest
        return np.stack(idx, axis=1)

    def global_ids(self):
        """(J,) GlobalID of every cell in local order: ``ix + iy*nX + iz*nX*nY`` in 3D
        (``Grid3D.cs:248``), ``ix*nY + iy`` in 2D (``Grid2D.cs:182``)."""
        ijk = self.cell_ijk().astype(np.int64)
        if self.dim == 2:
            return ijk[:, 0] * self.n[1] + ijk[:, 1]
        return ijk[:, 0] + self.n[0] * (ijk[:, 1] + self.n[1] * ijk[:, 2])


def Cartesian2DGrid(xNodes, yNodes, periodicX=False, periodicY=False, cell_order=C.CELLS_GENERATOR):
    return CartesianGrid([xNodes, yNodes], [periodicX, periodicY], cell_order)


def Cartesian3DGrid(xNodes, yNodes, zNodes, periodicX=False, periodicY=False, periodicZ=False,
                    cell_order=C.CELLS_GENERATOR):
    return CartesianGrid([xNodes, yNodes, zNodes], [periodicX, periodicY, periodicZ], cell_order)


def np_of(dim, k):
    return (k + 1) * (k + 2) // 2 if dim == 2 else (k + 1) * (k + 2) * (k + 3) // 6


class DGField:
    """A named DG field of a given degree on a grid (``SinglePhaseField``)."""

    def __init__(self, grid, degree, name):
        self.grid, self.degree, self.name = grid, int(degree), name

    @property
    def Np(self):
        return np_of(self.grid.dim, self.degree)


class CoordinateVector:
    """Coefficients of several fields in the cell-major layout
    ``j*N + fieldOffset[f] + n`` (``UnsetteledCoordinateMapping.cs:696-706``)."""

    def __init__(self, fields, data=None):
        self.fields = list(fields)
        self.grid = self.fields[0].grid
        self.per_cell = sum(f.Np for f in self.fields)
        n = self.grid.NoOfCells * self.per_cell
        self.data = np.zeros(n) if data is None else data
        if self.data.shape[0] != n:
            raise ValueError("coordinate vector has length %d, expected %d" % (self.data.shape[0], n))

    def field_view(self, f):
        """(J, Np) view of field f."""
        off = sum(x.Np for x in self.fields[:f])
        return self.data.reshape(self.grid.NoOfCells, self.per_cell)[:, off:off + self.fields[f].Np]


# ----------------------------------------------------------------------------- components


class _Component:
    ctype = None
    ArgumentOrdering = ()
    ParameterOrdering = None

    def params(self, dim):
        return []

    def fill(self, comp, cod_index, arg_index, dim):
        comp.type = self.ctype
        comp.codomain = cod_index
        comp.n_args = len(self.ArgumentOrdering)
        for i, a in enumerate(self.ArgumentOrdering):
            comp.args[i] = arg_index[a]
        for i, v in enumerate(self.params(dim)):
            comp.params[i] = float(v)


class ScalarTransportFlux(_Component):
    """ScalarTransportFlux / ScalarTransportFlux3D (``TransportFlux.cs:29-191``), upwind,
    with the velocity parameter fields constant (``velocity``)."""
    ctype = C.COMP_SCALAR_TRANSPORT_FLUX

    def __init__(self, velocity, ArgumentVarName="u"):
        self.velocity = [float(v) for v in velocity]
        self.ArgumentOrdering = (ArgumentVarName,)

    def params(self, dim):
        if len(self.velocity) != dim:
            raise ValueError("velocity has wrong dimension")
        return self.velocity


class SIPLaplace(_Component):
    """SIPLaplace (``ipLaplace.cs:30-269``) with ``Nu`` generalised to
    ``nu(u) = nu0 + nu2*u^2``. ``dirichlet=True`` uses ``g_D(x) = g0 + g1.x + g2.x^2``
    (componentwise squares) on every boundary edge, else Neumann with ``g_N = 0``."""
    ctype = C.COMP_SIP_LAPLACE

    def __init__(self, penalty_base, ArgumentVarName="u", nu0=1.0, nu2=0.0, dirichlet=True,
                 g0=0.0, g1=(0.0, 0.0, 0.0), g2=(0.0, 0.0, 0.0)):
        self.penalty_base, self.nu0, self.nu2 = float(penalty_base), float(nu0), float(nu2)
        self.dirichlet = bool(dirichlet)
        self.g0, self.g1, self.g2 = float(g0), list(g1) + [0.0] * (3 - len(g1)), list(g2) + [0.0] * (3 - len(g2))
        self.ArgumentOrdering = (ArgumentVarName,)

    def params(self, dim):
        return ([self.penalty_base, self.nu0, self.nu2, 0.0 if self.dirichlet else 1.0, self.g0]
                + self.g1[:3] + self.g2[:3])


class ConstantSource(_Component):
    """Constant volume source ``s * v`` (INonlinearSource)."""
    ctype = C.COMP_CONSTANT_SOURCE

    def __init__(self, value, ArgumentVarName="u"):
        self.value = float(value)
        self.ArgumentOrdering = (ArgumentVarName,)

    def params(self, dim):
        return [self.value]


class Material:
    """Ideal gas with ``HeatCapacityRatio`` gamma and reference ``MachNumber``."""

    def __init__(self, gamma=1.4, Mach=None):
        self.gamma = float(gamma)
        self.Mach = float(Mach) if Mach is not None else 1.0 / np.sqrt(self.gamma)


def _euler_args(dim):
    return tuple(["rho"] + ["m%d" % d for d in range(dim)] + ["rhoE"])


class OptimizedHLLCDensityFlux(_Component):
    """``Convection/OptimizedHLLCDensityFlux.cs``"""
    ctype = C.COMP_HLLC_DENSITY_FLUX

    def __init__(self, material, dim=3):
        self.material = material
        self.ArgumentOrdering = _euler_args(dim)

    def params(self, dim):
        return [self.material.gamma, self.material.Mach, 0.0]


class OptimizedHLLCMomentumFlux(OptimizedHLLCDensityFlux):
    """``Convection/OptimizedHLLCMomentumFlux.cs``"""
    ctype = C.COMP_HLLC_MOMENTUM_FLUX

    def __init__(self, material, component, dim=3):
        super().__init__(material, dim)
        self.component = int(component)

    def params(self, dim):
        return [self.material.gamma, self.material.Mach, float(self.component)]


class OptimizedHLLCEnergyFlux(OptimizedHLLCDensityFlux):
    """``Convection/OptimizedHLLCEnergyFlux.cs``"""
    ctype = C.COMP_HLLC_ENERGY_FLUX


class CNSMaterial:
    """Material and numerics of the CNS viscous terms (CNSControl / Material.cs): ideal gas
    gamma, Mach (default 1/sqrt(gamma): MachScaling = 1), Reynolds, Prandtl, bulk / shear
    viscosity ratio, Sutherland's law (S/T0 = 110.4/273.15, SutherlandLaw.cs) or mu = 1, and
    the SIPG penalty scaling."""

    def __init__(self, gamma=1.4, Mach=None, Reynolds=1.0, Prandtl=1.0, ViscosityRatio=0.0, sutherland=True,
                 sutherland_ratio=110.4 / 273.15, SIPGPenaltyScaling=1.0):
        self.gamma = float(gamma)
        self.Mach = float(Mach) if Mach is not None else 1.0 / np.sqrt(gamma)
        self.Re, self.Pr, self.alpha = float(Reynolds), float(Prandtl), float(ViscosityRatio)
        self.law = 1.0 if sutherland else 0.0
        self.suth, self.penalty = float(sutherland_ratio), float(SIPGPenaltyScaling)


class OptimizedSIPGDensityFlux(_Component):
    """``CNS/Diffusion/OptimizedSIPGDensityFlux.cs`` (no viscous density flux)."""
    ctype = C.COMP_CNS_SIPG_DENSITY_FLUX

    def __init__(self, material, dim=3):
        self.material = material
        self.ArgumentOrdering = _euler_args(dim)
        self.component = 0

    def params(self, dim):
        m = self.material
        return [m.gamma, m.Mach, m.Re, m.Pr, m.alpha, m.law, m.suth, m.penalty, float(self.component)]


class OptimizedSIPGMomentumFlux(OptimizedSIPGDensityFlux):
    """``CNS/Diffusion/OptimizedSIPGMomentumFlux.cs``, momentum component ``component``."""
    ctype = C.COMP_CNS_SIPG_MOMENTUM_FLUX

    def __init__(self, material, component, dim=3):
        super().__init__(material, dim)
        self.component = int(component)


class OptimizedSIPGEnergyFlux(OptimizedSIPGDensityFlux):
    """``CNS/Diffusion/OptimizedSIPGEnergyFlux.cs``."""
    ctype = C.COMP_CNS_SIPG_ENERGY_FLUX


# ----------------------------------------------------------------------------- operator


class _ComponentList(list):
    def Add(self, comp):
        self.append(comp)


class DifferentialOperator:
    def __init__(self, DomainVarNames, ParameterVarNames, CodomainVarNames, QuadOrderFunc_=None):
        self.DomainVar = list(DomainVarNames)
        self.ParameterVar = list(ParameterVarNames or [])
        self.CodomainVar = list(CodomainVarNames)
        self.QuadOrderFunction = QuadOrderFunc_ or QuadOrderFunc.NonLinear(2)
        self.EquationComponents = {c: _ComponentList() for c in self.CodomainVar}
        self.IsCommitted = False

    def Commit(self):
        if self.IsCommitted:
            raise RuntimeError("operator is already committed")
        for cod, comps in self.EquationComponents.items():
            for c in comps:
                for a in c.ArgumentOrdering:
                    if a not in self.DomainVar:
                        raise ValueError("component on '%s' uses unknown argument '%s'" % (cod, a))
        self.IsCommitted = True

    def descriptor(self, domain_degrees, codomain_degrees, dim):
        if not self.IsCommitted:
            raise RuntimeError("operator must be committed before an evaluator is created")
        d = C.OpDesc()
        d.n_domain = len(self.DomainVar)
        d.n_codomain = len(self.CodomainVar)
        for i, k in enumerate(domain_degrees):
            d.domain_degree[i] = int(k)
        for i, k in enumerate(codomain_degrees):
            d.codomain_degree[i] = int(k)
        d.quad_kind, d.quad_param = self.QuadOrderFunction
        arg_index = {n: i for i, n in enumerate(self.DomainVar)}
        n = 0
        for ci, cod in enumerate(self.CodomainVar):
            for comp in self.EquationComponents[cod]:
                if n >= C.MAX_COMPONENTS:
                    raise ValueError("too many components")
                comp.fill(d.components[n], ci, arg_index, dim)
                n += 1
        d.n_components = n
        return d

    def GetEvaluatorEx(self, DomainFields, ParameterMap, CodomainVarMap, device=0,
                       precision=C.PRECISION_FP64, check_nan=False, kernel=C.KERNEL_AUTO):
        """``DomainFields``: list of DGField (or a CoordinateVector); ``CodomainVarMap``:
        list of DGField of the codomain. ``ParameterMap`` must be empty (parameters are
        component constants on the device path)."""
        if ParameterMap:
            raise C.BosssError(C.ERR_BAD_ARG, "parameter fields are not supported by the device path")
        dom = DomainFields.fields if isinstance(DomainFields, CoordinateVector) else list(DomainFields)
        cod = CodomainVarMap.fields if isinstance(CodomainVarMap, CoordinateVector) else list(CodomainVarMap)
        if len(dom) != len(self.DomainVar) or len(cod) != len(self.CodomainVar):
            raise ValueError("mismatch between number of fields and operator variables")
        grid = dom[0].grid
        return Evaluator(self, grid, [f.degree for f in dom], [f.degree for f in cod],
                         DomainFields if isinstance(DomainFields, CoordinateVector) else None,
                         device, precision, check_nan, kernel)


def _solver_opts(rtol=None, atol=None, max_outer=None, restart=None, max_krylov=None, precond=1, inner_rtol=None,
                 precond_update=None):
    o = C.SolverOpts()
    o.precond_update = precond_update or 0
    o.rtol = rtol or 0.0
    o.atol = atol or 0.0
    o.max_outer = max_outer or 0
    o.restart = restart or 0
    o.max_krylov = max_krylov or 0
    o.precond = int(precond)
    o.inner_rtol = inner_rtol or 0.0
    return o


def _report(r):
    return {"outer_iters": r.outer_iters, "krylov_iters": r.krylov_iters, "converged": bool(r.converged),
            "residual0": r.residual0, "residual": r.residual}


class MultigridPreconditioner:
    """One V-cycle of ClassicMultigrid over the p-levels (LevelPmg) and aggregation levels of a
    scalar Jacobian (bosss_b200_pmg_*); ``apply_device`` takes device pointers."""

    def __init__(self, handle):
        self.handle = handle

    def info(self):
        npl, nhl, nc, direct = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64(), ctypes.c_int32()
        C.check(C.lib().bosss_b200_pmg_info(self.handle, ctypes.byref(npl), ctypes.byref(nhl), ctypes.byref(nc),
                                            ctypes.byref(direct)))
        return {"p_levels": npl.value, "h_levels": nhl.value, "coarsest": nc.value, "direct": bool(direct.value)}

    def apply_device(self, b, x, stream=None):
        C.check(C.lib().bosss_b200_pmg_apply_device(self.handle, C.ptr(b), C.ptr(x), stream))

    def Dispose(self):
        if self.handle:
            C.lib().bosss_b200_pmg_destroy(self.handle)
            self.handle = None

    __del__ = Dispose


class BlockMsrMatrix:
    """Device block-sparse matrix with dense cell blocks (``BlockMsrMatrix.cs:186``):
    ``SpMV(alpha, x, beta, y)`` is ``BlockMsrMatrix.SpMV`` (``:2554``)."""

    def __init__(self, handle):
        self.handle = handle
        nbr, nbc, br, bc, nnzb = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int64()
        C.check(C.lib().bosss_b200_bsr_get(handle, ctypes.byref(nbr), ctypes.byref(nbc), ctypes.byref(br),
                                           ctypes.byref(bc), ctypes.byref(nnzb), None, None, None))
        self.n_block_rows, self.n_block_cols = nbr.value, nbc.value
        self.row_block, self.col_block, self.nnz_blocks = br.value, bc.value, nnzb.value

    @classmethod
    def from_blocks(cls, n_block_rows, n_block_cols, row_ptr, col_idx, values, device=0):
        rp = np.ascontiguousarray(row_ptr, dtype=np.int64)
        ci = np.ascontiguousarray(col_idx, dtype=np.int32)
        v = np.ascontiguousarray(values, dtype=np.float64)
        if v.ndim != 3 or v.shape[0] != len(ci):
            raise ValueError("values must have shape (nnz_blocks, row_block, col_block)")
        h = ctypes.c_void_p()
        C.check(C.lib().bosss_b200_bsr_create(n_block_rows, n_block_cols, v.shape[1], v.shape[2], C.ptr(rp),
                                              C.ptr(ci), C.ptr(v), int(device), ctypes.byref(h)))
        return cls(h)

    def Dispose(self):
        if self.handle:
            C.lib().bosss_b200_bsr_destroy(self.handle)
            self.handle = None

    __del__ = Dispose

    def blocks(self):
        """(row_ptr, col_idx, values[nnz, row_block, col_block])."""
        rp = np.zeros(self.n_block_rows + 1, dtype=np.int64)
        ci = np.zeros(self.nnz_blocks, dtype=np.int32)
        v = np.zeros(self.nnz_blocks * self.row_block * self.col_block)
        C.check(C.lib().bosss_b200_bsr_get(self.handle, None, None, None, None, None, C.ptr(rp), C.ptr(ci), C.ptr(v)))
        return rp, ci, v.reshape(self.nnz_blocks, self.row_block, self.col_block)

    def SpMV(self, alpha, x, beta, y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        C.check(C.lib().bosss_b200_bsr_spmv(self.handle, alpha, C.ptr(x), beta, C.ptr(y)))
        return y

    def Solve(self, b, x=None, **kw):
        """FP32 GMRES in FP64 iterative refinement; returns (x, report)."""
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b) if x is None else np.array(x, dtype=np.float64, copy=True)
        o = _solver_opts(**kw)
        r = C.SolverReport()
        C.check(C.lib().bosss_b200_bsr_solve(self.handle, C.ptr(b), C.ptr(x), ctypes.byref(o), ctypes.byref(r)))
        return x, _report(r)


class Evaluator:
    """``IEvaluatorNonLin`` backed by one ``bosss_handle``."""

    def __init__(self, op, grid, dom_deg, cod_deg, bound, device, precision, check_nan, kernel=C.KERNEL_AUTO):
        self.handle = None
        self.op, self.grid = op, grid
        self.desc = op.descriptor(dom_deg, cod_deg, grid.dim)
        self.gdesc = grid.desc()
        opt = C.Options()
        opt.device, opt.precision, opt.check_nan = int(device), int(precision), int(bool(check_nan))
        opt.kernel = int(kernel)
        h = ctypes.c_void_p()
        C.check(C.lib().bosss_b200_create(ctypes.byref(self.desc), ctypes.byref(self.gdesc), ctypes.byref(opt),
                                          ctypes.byref(h)))
        self.handle = h
        nd, nc, nq = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
        C.check(C.lib().bosss_b200_get_sizes(h, ctypes.byref(nd), ctypes.byref(nc), ctypes.byref(nq)))
        self.n_domain, self.n_codomain, self.quad_nodes_1d = nd.value, nc.value, nq.value
        self.bound = bound
        self.time = 0.0

    # -- lifetime
    def Dispose(self):
        if self.handle:
            C.lib().bosss_b200_destroy(self.handle)
            self.handle = None

    __del__ = Dispose

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.Dispose()

    def kernel_info(self, mode=C.MODE_RESIDUAL):
        """(kernel path, launches per whole-grid call) of `mode`: 1 generic, 2 slab, 3 slab
        volume pass + face-once face kernels, 4 tensor-core volume + face terms."""
        k, n = ctypes.c_int32(), ctypes.c_int32()
        C.check(C.lib().bosss_b200_kernel_info(self.handle, int(mode), ctypes.byref(k), ctypes.byref(n)))
        return k.value, n.value

    # -- evaluation
    @staticmethod
    def _is_cuda(a):
        return hasattr(a, "is_cuda") and a.is_cuda

    def _stream(self):
        """The current torch stream; torch's legacy default stream (handle 0) is passed as
        cudaStreamLegacy, since a NULL stream selects the handle's own stream."""
        import torch
        s = torch.cuda.current_stream().cuda_stream
        return ctypes.c_void_p(s if s else C.CUDA_STREAM_LEGACY)

    def Evaluate(self, alpha, beta, output, U=None):
        """``output = beta*output + alpha*Op(U)``; ``U`` defaults to the bound domain
        fields. numpy arrays go through the host entry point, CUDA tensors through the
        device-resident one (enqueued on the current torch stream)."""
        if U is None:
            if self.bound is None:
                raise ValueError("no domain fields bound")
            U = self.bound.data
        out = output.data if isinstance(output, CoordinateVector) else output
        if len(U) != self.n_domain or len(out) != self.n_codomain:
            raise C.BosssError(C.ERR_BAD_ARG, "wrong vector length")   # DifferentialOperator.cs:1590-1591
        if self._is_cuda(U):
            C.check(C.lib().bosss_b200_evaluate_device(self.handle, alpha, beta, C.ptr(U), C.ptr(out),
                                                       self.time, self._stream()))
        else:
            U = np.ascontiguousarray(U, dtype=np.float64)
            C.check(C.lib().bosss_b200_evaluate(self.handle, alpha, beta, C.ptr(U), C.ptr(out), self.time))
        return out

    def jvp(self, U, V, out=None):
        """J(U) V (directional derivative)."""
        if self._is_cuda(U):
            import torch
            out = torch.empty(self.n_codomain, dtype=torch.float64, device=U.device) if out is None else out
            C.check(C.lib().bosss_b200_jvp_device(self.handle, C.ptr(U), C.ptr(V), C.ptr(out), self.time,
                                                  self._stream()))
            return out
        U = np.ascontiguousarray(U, dtype=np.float64)
        V = np.ascontiguousarray(V, dtype=np.float64)
        out = np.empty(self.n_codomain) if out is None else out
        C.check(C.lib().bosss_b200_jvp(self.handle, C.ptr(U), C.ptr(V), C.ptr(out), self.time))
        return out

    def ComputeJacobian(self, U):
        """Exact Jacobian at U as a device BlockMsrMatrix (cell blocks: self + face neighbours)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        h = ctypes.c_void_p()
        C.check(C.lib().bosss_b200_compute_jacobian(self.handle, C.ptr(U), self.time, ctypes.byref(h)))
        return BlockMsrMatrix(h)

    def Multigrid(self, A):
        """Multigrid V-cycle preconditioner of the Jacobian A (from ComputeJacobian)."""
        h = ctypes.c_void_p()
        C.check(C.lib().bosss_b200_pmg_create(self.handle, A.handle, ctypes.byref(h)))
        return MultigridPreconditioner(h)

    def NewtonSolve(self, U0, **kw):
        """Matrix-free Newton-GMRES for Op(U) = 0; returns (U, report)."""
        U = np.array(U0, dtype=np.float64, copy=True)
        o = _solver_opts(**kw)
        r = C.SolverReport()
        C.check(C.lib().bosss_b200_newton_solve(self.handle, C.ptr(U), self.time, ctypes.byref(o), ctypes.byref(r)))
        return U, _report(r)

    def boundary_nodes(self):
        """Coordinates (n, D) of the boundary face nodes of the boundary-state table."""
        n = ctypes.c_int64()
        C.check(C.lib().bosss_b200_boundary_nodes(self.handle, ctypes.byref(n), None))
        xyz = np.zeros(n.value * self.grid.dim)
        if n.value:
            C.check(C.lib().bosss_b200_boundary_nodes(self.handle, ctypes.byref(n), C.ptr(xyz)))
        return xyz.reshape(n.value, self.grid.dim)

    def SetBoundaryState(self, state):
        """Outer state (n_nodes, n_domain) at the boundary face nodes, what the C# side's
        boundary-condition map returns there (e.g. SupersonicInlet.GetBoundaryState)."""
        a = np.ascontiguousarray(state, dtype=np.float64)
        C.check(C.lib().bosss_b200_set_boundary_state(self.handle, C.ptr(a)))

    def SetBoundaryKinds(self, kinds):
        """Boundary-condition kind per boundary face node (HLLC): 0 prescribed state from the
        table, 1 supersonic outlet (inner state), 2 adiabatic slip wall (normal momentum
        reflected)."""
        a = np.ascontiguousarray(kinds, dtype=np.int32)
        C.check(C.lib().bosss_b200_set_boundary_kinds(self.handle, C.ptr(a)))

    def residual_vjp(self, U, W, R=None, G=None, alpha=1.0, beta=0.0):
        """Host arrays: ``R = beta*R + alpha*Op(U)`` and ``G = J(U)^T W`` in one pipelined call
        (U and W cross PCIe once). Returns (R, G)."""
        U = np.ascontiguousarray(U, dtype=np.float64)
        W = np.ascontiguousarray(W, dtype=np.float64)
        R = np.zeros(self.n_codomain) if R is None else R
        G = np.empty(self.n_domain) if G is None else G
        C.check(C.lib().bosss_b200_residual_vjp(self.handle, alpha, beta, C.ptr(U), C.ptr(R), C.ptr(W), C.ptr(G),
                                                self.time))
        return R, G

    def vjp(self, U, W, out=None):
        """J(U)^T W (adjoint product)."""
        if self._is_cuda(U):
            import torch
            out = torch.empty(self.n_domain, dtype=torch.float64, device=U.device) if out is None else out
            C.check(C.lib().bosss_b200_vjp_device(self.handle, C.ptr(U), C.ptr(W), C.ptr(out), self.time,
                                                  self._stream()))
            return out
        U = np.ascontiguousarray(U, dtype=np.float64)
        W = np.ascontiguousarray(W, dtype=np.float64)
        out = np.empty(self.n_domain) if out is None else out
        C.check(C.lib().bosss_b200_vjp(self.handle, C.ptr(U), C.ptr(W), C.ptr(out), self.time))
        return out


class BatchEvaluator:
    """Independent operator instances evaluated by one persistent launch per mode.

    ``problems``: list of objects with ``descs()`` (operator and grid descriptors), e.g.
    :class:`bosss_b200.problems.Problem`. Vectors are the concatenation of the
    instances' vectors; ``offsets`` gives the instance boundaries."""

    def __init__(self, problems, device=0, kernel=C.KERNEL_AUTO):
        self.handle = None
        descs = [p.descs() for p in problems]
        self.n = len(descs)
        self._ops = (C.OpDesc * self.n)(*[d[0] for d in descs])
        self._grids = (C.GridDesc * self.n)(*[d[1] for d in descs])
        opt = C.Options()
        opt.device = int(device)
        opt.kernel = int(kernel)   # tile kernel: 0 automatic, 1 generic tiles, 2 slab tiles where possible
        h = ctypes.c_void_p()
        C.check(C.lib().bosss_b200_batch_create(self.n, ctypes.byref(self._ops), ctypes.byref(self._grids),
                                                ctypes.byref(opt), ctypes.byref(h)))
        self.handle = h
        self.dom_offsets = np.zeros(self.n + 1, dtype=np.int64)
        self.cod_offsets = np.zeros(self.n + 1, dtype=np.int64)
        C.check(C.lib().bosss_b200_batch_get_sizes(h, C.ptr(self.dom_offsets), C.ptr(self.cod_offsets)))

    def Dispose(self):
        if self.handle:
            C.lib().bosss_b200_batch_destroy(self.handle)
            self.handle = None

    __del__ = Dispose

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.Dispose()

    def evaluate(self, mode, U, V=None, out=None, alpha=1.0, beta=0.0):
        """Host or CUDA-tensor buffers (device path enqueued on the current torch stream)."""
        nout = int(self.dom_offsets[-1] if mode == C.MODE_VJP else self.cod_offsets[-1])
        if hasattr(U, "is_cuda") and U.is_cuda:
            import torch
            out = torch.zeros(nout, dtype=torch.float64, device=U.device) if out is None else out
            s = torch.cuda.current_stream().cuda_stream
            C.check(C.lib().bosss_b200_batch_evaluate_device(self.handle, mode, alpha, beta, C.ptr(U), C.ptr(V),
                                                             C.ptr(out), 0.0,
                                                             ctypes.c_void_p(s if s else C.CUDA_STREAM_LEGACY)))
            return out
        U = np.ascontiguousarray(U, dtype=np.float64)
        V = None if V is None else np.ascontiguousarray(V, dtype=np.float64)
        out = np.zeros(nout) if out is None else out
        C.check(C.lib().bosss_b200_batch_evaluate(self.handle, mode, alpha, beta, C.ptr(U), C.ptr(V), C.ptr(out), 0.0))
        return out

    def solve(self, dt, b, x=None, U=None, transpose=False, **kw):
        """Per-instance implicit-step systems (I/dt_i + J_i) x_i = b_i (``transpose``: the
        adjoint systems), FP32 GMRES inside FP64 refinement; CUDA tensors. ``dt``: one value or
        one per instance. Returns (x, reports)."""
        import torch
        dts = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (self.n,)))
        x = torch.zeros_like(b) if x is None else x
        o = _solver_opts(**kw)
        reps = (C.SolverReport * self.n)()
        torch.cuda.synchronize()
        C.check(C.lib().bosss_b200_batch_solve(self.handle, int(bool(transpose)), C.ptr(dts), C.ptr(U), C.ptr(b),
                                               C.ptr(x), ctypes.byref(o), ctypes.cast(reps, ctypes.c_void_p)))
        return x, [_report(r) for r in reps]

    def capture(self, U, W, R, G):
        """Capture residual R = Op(U) and adjoint G = J^T W (CUDA tensors) into a CUDA graph."""
        C.check(C.lib().bosss_b200_batch_capture(self.handle, C.ptr(U), C.ptr(W), C.ptr(R), C.ptr(G), 0.0))

    def replay(self, stream=None):
        import torch
        s = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
        C.check(C.lib().bosss_b200_batch_replay(self.handle, ctypes.c_void_p(s if s else C.CUDA_STREAM_LEGACY)))

    def autotune(self, U, W, R, G, table_path=None):
        C.check(C.lib().bosss_b200_batch_autotune(self.handle, C.ptr(U), C.ptr(W), C.ptr(R), C.ptr(G),
                                                  table_path.encode() if table_path else None))

    SCHEDULES = {0: "fifo", 1: "lpt", 2: "classes"}

    def tiles(self, K, Q):
        """(tiles per work item of the (K, Q) class, schedule: "lpt" | "fifo" | "classes")."""
        t, sched = ctypes.c_int32(), ctypes.c_int32()
        C.check(C.lib().bosss_b200_batch_tiles(self.handle, K, Q, ctypes.byref(t), ctypes.byref(sched)))
        return t.value, BatchEvaluator.SCHEDULES[sched.value]


class XdgEvaluator:
    """Per-species bulk evaluation of an XDG operator (``XEvaluatorNonlin.Evaluate``, bulk
    part): ``opA`` / ``opB`` are the committed bulk operators of species A (phi < 0) and B
    (phi >= 0), e.g. ``XLaplace_Bulk`` = :class:`SIPLaplace` with nu = mu_s; the level set is a
    sphere ``phi = |x - c| - r``. Vectors are full-grid species frames."""

    def __init__(self, opA, opB, grid, degree, center, radius, device=0, cut_nodes_1d=5, fallback_nodes_1d=9,
                 moment_degree=-1, subdivision=8, kernel=C.KERNEL_AUTO, rule=C.XDG_RULE_MOMENT_FITTING):
        self.handle = None
        self.grid, self.degree = grid, degree
        self.descA = opA.descriptor([degree], [degree], grid.dim)
        self.descB = opB.descriptor([degree], [degree], grid.dim)
        self.gdesc = grid.desc()
        ls = C.LevelSetDesc()
        ls.type = C.LEVELSET_SPHERE
        for i, v in enumerate(list(center) + [radius]):
            ls.params[i] = float(v)
        xo = C.XdgOpts()
        xo.cut_nodes_1d, xo.fallback_nodes_1d = cut_nodes_1d, fallback_nodes_1d
        xo.moment_degree, xo.subdivision = moment_degree, subdivision
        xo.rule = int(rule)
        opt = C.Options()
        opt.device = int(device)
        opt.kernel = int(kernel)
        h = ctypes.c_void_p()
        C.check(C.lib().bosss_b200_xdg_create(ctypes.byref(self.descA), ctypes.byref(self.descB),
                                              ctypes.byref(self.gdesc), ctypes.byref(ls), ctypes.byref(xo),
                                              ctypes.byref(opt), ctypes.byref(h)))
        self.handle = h
        self.n = grid.NoOfCells * np_of(grid.dim, degree)

    def Dispose(self):
        if self.handle:
            C.lib().bosss_b200_xdg_destroy(self.handle)
            self.handle = None

    __del__ = Dispose

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.Dispose()

    def info(self, species):
        v = [ctypes.c_int64() for _ in range(3)] + [ctypes.c_int32() for _ in range(3)] + [ctypes.c_double()]
        C.check(C.lib().bosss_b200_xdg_info(self.handle, species, *[ctypes.byref(x) for x in v]))
        keys = ["cells", "cut_cells", "cut_faces", "min_nodes", "max_nodes", "min_degree", "max_fit_residual"]
        return dict(zip(keys, [x.value for x in v]))

    def rules(self, species):
        cnt = (ctypes.c_int64 * 2)()
        C.check(C.lib().bosss_b200_xdg_get_rules(self.handle, species, cnt, None, None, None, None, None, None))
        ni, nn = cnt[0], cnt[1]
        J = self.grid.NoOfCells
        info = np.zeros(ni * 5, dtype=np.int64)
        offs = np.zeros(ni + 1, dtype=np.int64)
        nodes = np.zeros(nn * 3)
        w = np.zeros(nn)
        vf = np.zeros(J, dtype=np.uint8)
        ff = np.zeros(J * 6, dtype=np.uint8)
        C.check(C.lib().bosss_b200_xdg_get_rules(self.handle, species, cnt, C.ptr(info), C.ptr(offs), C.ptr(nodes),
                                                 C.ptr(w), C.ptr(vf), C.ptr(ff)))
        mom = np.zeros(ni * 35)
        C.check(C.lib().bosss_b200_xdg_get_moments(self.handle, species, C.ptr(mom)))
        return {"info": info.reshape(ni, 5), "offsets": offs, "nodes": nodes.reshape(nn, 3), "weights": w,
                "vol_flags": vf, "face_flags": ff, "moments": mom.reshape(ni, 35)}

    def length_scales(self, species):
        """The species' cell length scales of the SIP penalty (``CoefficientSet.CellLengthScales``
        of the species); NaN on cells without the species."""
        out = np.zeros(self.grid.NoOfCells)
        C.check(C.lib().bosss_b200_xdg_get_length_scales(self.handle, species, C.ptr(out)))
        return out

    def set_length_scales(self, species, length_scales=None):
        """The caller's length scales (e.g. agglomerated ones); None restores the defaults."""
        if length_scales is None:
            C.check(C.lib().bosss_b200_xdg_set_length_scales(self.handle, species, None))
            return
        a = np.ascontiguousarray(length_scales, dtype=np.float64)
        if a.shape != (self.grid.NoOfCells,):
            raise C.BosssError(C.ERR_BAD_ARG, "one length scale per cell")
        C.check(C.lib().bosss_b200_xdg_set_length_scales(self.handle, species, C.ptr(a)))

    def Evaluate(self, species, alpha, beta, output, U):
        if hasattr(U, "is_cuda") and U.is_cuda:
            import torch
            s = torch.cuda.current_stream().cuda_stream
            C.check(C.lib().bosss_b200_xdg_evaluate_device(self.handle, species, alpha, beta, C.ptr(U), C.ptr(output),
                                                           0.0, ctypes.c_void_p(s if s else C.CUDA_STREAM_LEGACY)))
            return output
        U = np.ascontiguousarray(U, dtype=np.float64)
        C.check(C.lib().bosss_b200_xdg_evaluate(self.handle, species, alpha, beta, C.ptr(U), C.ptr(output), 0.0))
        return output

    # ---- level-set interface term (XLaplace_Interface through NECQuadratureLevelSet)
    SWIP, SIP = 0, 1   # XLaplace_Interface.Mode, reference order

    def SetInterface(self, muA, muB, penalty_base, mode=SIP, nodes_1d=6):
        """Adds the interface component ``XLaplace_Interface(muA, muB, penalty_base, mode)``
        (XLaplace.cs:214-220) and builds the surface rules of the sphere in the cut cells."""
        C.check(C.lib().bosss_b200_xdg_interface_setup(self.handle, float(muA), float(muB), float(penalty_base),
                                                       int(mode), int(nodes_1d)))

    def interface_rules(self):
        """Surface rules: cut cells, node offsets, nodes (reference coordinates of the cell),
        weights (physical surface measure) and unit normals from A into B."""
        cnt = (ctypes.c_int64 * 2)()
        C.check(C.lib().bosss_b200_xdg_interface_get_rules(self.handle, cnt, None, None, None, None, None))
        nc, nq = cnt[0], cnt[1]
        cells = np.zeros(nc, dtype=np.int64)
        offs = np.zeros(nc + 1, dtype=np.int64)
        nodes, w, nrm = np.zeros(nq * 3), np.zeros(nq), np.zeros(nq * 3)
        C.check(C.lib().bosss_b200_xdg_interface_get_rules(self.handle, cnt, C.ptr(cells), C.ptr(offs), C.ptr(nodes),
                                                           C.ptr(w), C.ptr(nrm)))
        return {"cells": cells, "offsets": offs, "nodes": nodes.reshape(nq, 3), "weights": w,
                "normals": nrm.reshape(nq, 3)}

    def EvaluateInterface(self, alpha, UA, UB, outA, outB):
        """outA += alpha * (interface term tested with species A), outB likewise."""
        if hasattr(UA, "is_cuda") and UA.is_cuda:
            import torch
            s = torch.cuda.current_stream().cuda_stream
            C.check(C.lib().bosss_b200_xdg_interface_evaluate_device(
                self.handle, alpha, C.ptr(UA), C.ptr(UB), C.ptr(outA), C.ptr(outB),
                ctypes.c_void_p(s if s else C.CUDA_STREAM_LEGACY)))
            return outA, outB
        UA = np.ascontiguousarray(UA, dtype=np.float64)
        UB = np.ascontiguousarray(UB, dtype=np.float64)
        C.check(C.lib().bosss_b200_xdg_interface_evaluate(self.handle, alpha, C.ptr(UA), C.ptr(UB), C.ptr(outA),
                                                          C.ptr(outB)))
        return outA, outB
