"""Explicit Runge-Kutta time stepping around the device evaluator.

Mirrors ``BoSSS.Solution.TimeStepping``:

* ``RungeKuttaScheme(a, b, c)`` with the consistency checks of its constructor and the
  named tableaus (``RungeKuttaScheme.cs:55-420``); ``RungeKuttaSchemes`` +
  ``RungeKutta.SchemeFactory`` (``RungeKutta.cs:199-226``);
* ``RungeKutta(scheme, evaluator)`` with ``Perform(dt)`` (``RungeKutta.cs:242-291``):
  ``k_s = Op(u_s)``, ``u_s = y0 - dt*sum_r a[s,r] k_r`` (``PerformStage``, ``:300-313``),
  ``y1 = y0 - dt*sum_s b[s] k_s``; the change rate is ``Evaluate(1, 1, k)`` into a cleared
  ``k`` (``ExplicitEuler.ComputeChangeRate``, ``ExplicitEuler.cs:223-229``);
* ``ExplicitEuler(evaluator)`` (``ExplicitEuler.cs:293-307``): ``u -= dt*Op(u)``.

Every stage runs on the GPU through ``bosss_b200_rk_steps`` /
``bosss_b200_rk_steps_device`` (one residual launch and one fused stage-combination launch per
stage, a step captured into a CUDA graph). Time-step constraints (``CalculateTimeStep``) and
the ``OnAfterFieldUpdate`` filter hook have no device counterpart: ``dt`` is the caller's.
"""
import ctypes

import numpy as np

from . import _capi as C


class RungeKuttaScheme:
    """Butcher tableau of an explicit Runge-Kutta scheme (``RungeKuttaScheme.cs:55-100``)."""

    def __init__(self, a, b, c):
        a = np.array(a, dtype=np.float64)
        b = np.array(b, dtype=np.float64).ravel()
        c = np.array(c, dtype=np.float64).ravel()
        S = c.size
        if a.ndim != 2 or a.shape[0] != a.shape[1] or a.shape[0] != S or b.size != S:
            raise ValueError("inconsistent Butcher tableau shapes")
        if abs(b.sum() - 1.0) > 1e-12:
            raise ValueError("weights b must sum to 1")
        if np.any(np.abs(a.sum(axis=1) - c) > 1e-12):
            raise ValueError("row sums of a must equal c")
        self.a, self.b, self.c = a, b, c

    @property
    def Stages(self):
        return self.c.size

    @property
    def IsExplicit(self):
        return not np.any(np.triu(self.a) != 0.0)

    # named tableaus (the classical published schemes)
    @staticmethod
    def ExplicitEuler():
        return RungeKuttaScheme([[0.0]], [1.0], [0.0])

    @staticmethod
    def ExplicitEuler2():
        """Two explicit Euler half steps (first order)."""
        return RungeKuttaScheme([[0, 0], [0.5, 0]], [0.5, 0.5], [0, 0.5])

    @staticmethod
    def Middlepoint():
        return RungeKuttaScheme([[0, 0], [0.5, 0]], [0, 1], [0, 0.5])

    @staticmethod
    def Heun2():
        return RungeKuttaScheme([[0, 0], [1, 0]], [0.5, 0.5], [0, 1])

    @staticmethod
    def Heun():
        """Heun's third-order scheme."""
        return RungeKuttaScheme([[0, 0, 0], [1 / 3, 0, 0], [0, 2 / 3, 0]], [0.25, 0, 0.75], [0, 1 / 3, 2 / 3])

    @staticmethod
    def RungeKutta3():
        """Kutta's third-order scheme."""
        return RungeKuttaScheme([[0, 0, 0], [0.5, 0, 0], [-1, 2, 0]], [1 / 6, 2 / 3, 1 / 6], [0, 0.5, 1])

    @staticmethod
    def TVD3():
        """Shu-Osher third-order TVD scheme in Butcher form."""
        return RungeKuttaScheme([[0, 0, 0], [1, 0, 0], [0.25, 0.25, 0]], [1 / 6, 1 / 6, 2 / 3], [0, 1, 0.5])

    @staticmethod
    def RungeKutta1901():
        """The classical fourth-order scheme."""
        return RungeKuttaScheme([[0, 0, 0, 0], [0.5, 0, 0, 0], [0, 0.5, 0, 0], [0, 0, 1, 0]],
                                [1 / 6, 2 / 6, 2 / 6, 1 / 6], [0, 0.5, 0.5, 1])

    @staticmethod
    def ThreeOverEight():
        """Kutta's 3/8 rule."""
        return RungeKuttaScheme([[0, 0, 0, 0], [1 / 3, 0, 0, 0], [-1 / 3, 1, 0, 0], [1, -1, 1, 0]],
                                [1 / 8, 3 / 8, 3 / 8, 1 / 8], [0, 1 / 3, 2 / 3, 1])

    @staticmethod
    def SSP54():
        """Five-stage fourth-order strong-stability-preserving scheme (Spiteri and Ruuth, 2002)."""
        a = np.zeros((5, 5))
        a[1, 0] = 0.39175222657188905833
        a[2, :2] = [0.21766909626116921036, 0.36841059305037202075]
        a[3, :3] = [0.08269208665781075441, 0.13995850219189573938, 0.25189177427169263984]
        a[4, :4] = [0.06796628363711496324, 0.11503469850463199467, 0.20703489859738471851,
                    0.54497475022851992204]
        b = [0.14681187608478644956, 0.24848290944497614757, 0.10425883033198029567, 0.27443890090134945681,
             0.22600748323690765039]
        return RungeKuttaScheme(a, b, a.sum(axis=1))


class RungeKuttaSchemes:
    """Names accepted by :meth:`RungeKutta.SchemeFactory` (``RungeKutta.cs:199-226``)."""
    ExplicitEuler = "ExplicitEuler"
    Heun = "Heun"
    Middlepoint = "Middlepoint"
    RungeKutta1901 = "RungeKutta1901"
    ThreeOverEight = "ThreeOverEight"
    TVD3 = "TVD3"


class RungeKutta:
    """Explicit Runge-Kutta time stepper over one device evaluator (square operator).

    ``evaluator``: from ``DifferentialOperator.GetEvaluatorEx``; ``fields``: the
    :class:`CoordinateVector` stepped in place (default: the evaluator's bound domain fields).
    """

    MAX_STAGES = 8

    @staticmethod
    def SchemeFactory(scheme):
        if scheme not in (RungeKuttaSchemes.ExplicitEuler, RungeKuttaSchemes.Heun, RungeKuttaSchemes.Middlepoint,
                          RungeKuttaSchemes.RungeKutta1901, RungeKuttaSchemes.ThreeOverEight,
                          RungeKuttaSchemes.TVD3):
            raise NotImplementedError(scheme)
        return getattr(RungeKuttaScheme, scheme)()

    def __init__(self, scheme, evaluator, fields=None):
        if isinstance(scheme, str):
            scheme = RungeKutta.SchemeFactory(scheme)
        if not scheme.IsExplicit:
            raise ValueError("only explicit schemes are supported")
        if scheme.Stages > RungeKutta.MAX_STAGES:
            raise ValueError("at most %d stages" % RungeKutta.MAX_STAGES)
        if evaluator.n_domain != evaluator.n_codomain:
            raise ValueError("time stepping needs a square operator")
        self.Scheme = scheme
        self.Evaluator = evaluator
        self.CurrentState = fields if fields is not None else evaluator.bound
        self.Time = 0.0
        self._a = np.ascontiguousarray(scheme.a.ravel())
        self._b = np.ascontiguousarray(scheme.b)
        self._c = np.ascontiguousarray(scheme.c)
        self._work = None

    def work_size(self):
        n = ctypes.c_int64()
        C.check(C.lib().bosss_b200_rk_work_size(self.Evaluator.handle, self.Scheme.Stages, ctypes.byref(n)))
        return n.value

    def Perform(self, dt, nsteps=1):
        """Advance the host state ``CurrentState`` by ``nsteps`` steps of size ``dt``; returns dt."""
        U = self.CurrentState
        U = U if isinstance(U, np.ndarray) else U.data
        if not (isinstance(U, np.ndarray) and U.dtype == np.float64 and U.flags.c_contiguous):
            raise ValueError("the host state must be a contiguous float64 array")
        C.check(C.lib().bosss_b200_rk_steps(self.Evaluator.handle, self.Scheme.Stages, C.ptr(self._a),
                                            C.ptr(self._b), C.ptr(self._c), float(dt), int(nsteps),
                                            float(self.Time), C.ptr(U)))
        self.Time += nsteps * dt
        return dt

    def PerformDevice(self, U, dt, nsteps=1, use_graph=True):
        """Advance the CUDA tensor ``U`` in place (enqueued on the current torch stream)."""
        import torch
        n = self.work_size()
        if self._work is None or self._work.numel() < n or self._work.device != U.device:
            self._work = torch.empty(n, dtype=torch.float64, device=U.device)
        C.check(C.lib().bosss_b200_rk_steps_device(self.Evaluator.handle, self.Scheme.Stages, C.ptr(self._a),
                                                   C.ptr(self._b), C.ptr(self._c), float(dt), int(nsteps),
                                                   float(self.Time), C.ptr(U), C.ptr(self._work),
                                                   int(bool(use_graph)), self.Evaluator._stream()))
        self.Time += nsteps * dt
        return U


class ExplicitEuler(RungeKutta):
    """``ExplicitEuler.Perform`` (``ExplicitEuler.cs:293-307``): ``u <- u - dt*Op(u)``."""

    def __init__(self, evaluator, fields=None):
        super().__init__(RungeKuttaScheme.ExplicitEuler(), evaluator, fields)
