"""Drop-in density-matrix propagators running on B200.

* ``RhoVNeumannCUDA1D`` -- rho_vneumann_cuda_1d.py:15 (von Neumann equation)
* ``RhoBlochCUDA1D``    -- rho_bloch_cuda_1d.py:9    (Bloch equation for rho)

rho[i][j] = <x'_i| rho |x_j> lives on the GPU as a complex torch tensor
(complex128 by default, complex64 with ``precision="float32"``).  A step is
two fused passes of libfastwigner: a row pass (inverse FFT along x, exp(V),
observables, exp(V) of the next step, FFT along x) and a column pass (FFT
along x', exp(K), inverse FFT).  exp(V) and exp(K) are separable,
u(x) conj(u(x')), so the passes read two length-N vectors instead of N x N
tables.  The per-step trace normalisation is applied lazily in the next pass.
Observables Tr[rho g(p)] are evaluated in the row pass as
sum_ij rho_ij G[(i - j) mod N] with G = ifft(g(P)) -- the same number the
reference gets from row FFT, multiply, row inverse FFT and a trace
(rho_vneumann_cuda_1d.py:452-472).
"""
from __future__ import annotations

import ctypes
from types import FunctionType, MethodType

import numpy as np
import torch

from . import _lib, cexpr
from ._device import DeviceArray, ptr, require_cuda, stream_handle, to_device
from ._lib import FW_F32, FW_F64, FastWignerError, RhoDesc, RhoFactor, check
from .wigner import _bind_kwargs, _require

c_vp, c_ll, c_int, c_dbl = ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_double


def _factor(s=1.0, u=None, w=None, tab=None, shear=None, sign=False):
    f = RhoFactor()
    f.on = 1
    s = complex(s)
    f.s_re, f.s_im = s.real, s.imag
    f.u, f.w, f.tab = ptr(u), ptr(w), ptr(tab)
    if shear is not None:
        f.shear_c, f.shear_a, f.shear_b, f.shear_dx, f.shear_dp = shear
    f.sign = 1 if sign else 0
    return f


class RhoVNeumannCUDA1D:
    """Split-operator von Neumann propagator for rho(x, x', t) with C-string
    Hamiltonian H = K(P, t) + V(X, t) (drop-in for rho_vneumann_cuda_1d.py:15)."""

    _chunk = 512

    def __init__(self, **kwargs):
        _bind_kwargs(self, kwargs)
        _require(self, "X_gridDIM", "Coordinate grid size (X_gridDIM) was not specified")
        _require(self, "X_amplitude", "Coordinate grid range (X_amplitude) was not specified")
        _require(self, "V", "Potential energy (V) was not specified")
        _require(self, "K", "Momentum dependence (K) was not specified")
        _require(self, "dt", "Time-step (dt) was not specified")
        try:
            self.t
        except AttributeError:
            print("Warning: Initial time (t) was not specified, thus it is set to zero.")
            self.t = 0.0
        self.t = float(self.t)
        self.hbar = float(getattr(self, "hbar", 1.0))
        prec = str(getattr(self, "precision", "float64"))
        if prec not in ("float64", "float32"):
            raise ValueError("precision must be 'float64' or 'float32'")
        self.precision = prec
        f64 = prec == "float64"
        self._ct = torch.complex128 if f64 else torch.complex64
        self._rt = torch.float64 if f64 else torch.float32
        self._code = FW_F64 if f64 else FW_F32
        N = self.N = int(self.X_gridDIM)
        # grids (rho_vneumann_cuda_1d.py:94-110)
        self.dX = 2.0 * self.X_amplitude / N
        self.X = np.linspace(-self.X_amplitude, self.X_amplitude - self.dX, N)
        self.P = np.fft.fftfreq(N, self.dX / (2 * np.pi))
        self.dP = self.P[1] - self.P[0]
        self.P_wigner = self.P / np.sqrt(2.0)
        self.X_wigner = self.X / np.sqrt(2.0)
        self.wigner_dxdp = (self.X_wigner[1] - self.X_wigner[0]) * (self.P_wigner[1] - self.P_wigner[0])
        self.P_wigner = np.fft.fftshift(self.P_wigner)[:, np.newaxis]
        self.X_wigner = self.X_wigner[np.newaxis, :]
        j = np.arange(N)
        self._Xk = self.dX * (j - 0.5 * N)
        self._Pk = self.dP * ((j + N // 2) % N - 0.5 * N)
        kw = {k: v for k, v in kwargs.items() if k != "t"}
        kw.update(dX=self.dX, dP=self.dP)
        self.cuda_consts = cexpr.cuda_consts(kw, user_consts=getattr(self, "consts", ""))
        self.functions = getattr(self, "functions", "")
        exprs = {"fw_V": "V(X, t)", "fw_K": "K(P, t)"}
        self._bx_src = getattr(self, "abs_boundary_x", None)
        self._bp_src = getattr(self, "abs_boundary_p", None)
        if self._bx_src is not None:
            exprs["fw_bx"] = self._bx_src
        if self._bp_src is not None:
            exprs["fw_bp"] = self._bp_src
        try:
            self.diff_K
            self.diff_V
            self.isEhrenfest = True
            exprs.update(fw_dV=self.diff_V, fw_dK=self.diff_K)
        except AttributeError:
            self.isEhrenfest = False
        self.device = require_cuda()
        self._lib = _lib.load()
        self._mod = cexpr.ExprModule(self.cuda_consts, self.functions, exprs, K=self.K, V=self.V)
        self._observables = {}
        self._plan = c_vp()
        check(self._lib.fw_rho_plan_create(N, 1, self._code, ctypes.byref(self._plan)), "fw_rho_plan_create")
        self._nparts = self._lib.fw_rho_num_parts(self._plan)
        self.rho_t = torch.zeros((N, N), dtype=self._ct, device=self.device)
        self._tmp = torch.empty_like(self.rho_t)
        self._v_td = self._probe("fw_V", X=self._Xk)
        self._k_td = self._probe("fw_K", P=self._Pk)
        self._bx = self._table("fw_bx") if self._bx_src is not None else None
        self._bp = self._table("fw_bp", p=True) if self._bp_src is not None else None
        if self.isEhrenfest:
            self.X_average, self.P_average = [], []
            self.X_average_RHS, self.P_average_RHS = [], []
            self.hamiltonian_average = []
            self.wigner_time = []
            self._w_td = self._v_td or self._k_td or self._probe("fw_dV", X=self._Xk) or \
                self._probe("fw_dK", P=self._Pk)
        self._vec_cache = {}

    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                self._lib.fw_rho_plan_destroy(plan)
            except Exception:
                pass
            self._plan = None

    # -- helpers ------------------------------------------------------------
    def _probe(self, name, **c):
        a = self._mod.eval(name, self.N, t=0.0, **c)
        b = self._mod.eval(name, self.N, t=1.2345678, **c)
        return not torch.equal(a, b)

    def _table(self, name, p=False):
        N = self.N
        i = np.repeat(np.arange(N), N)
        j = np.tile(np.arange(N), N)
        g = self._Pk if p else self._Xk
        kw = dict(P=g[j], P_prime=g[i]) if p else dict(X=g[j], X_prime=g[i])
        v = self._mod.eval(name, N * N, t=self.t, i=i, j=j, indexTotal=j + i * N, **kw)
        return v.view(N, N).to(self._rt).contiguous()

    def _cvec(self, z):
        return to_device(np.asarray(z), self._ct, self.device)

    def _phase_vectors(self, t):
        """u, w for exp(V) and exp(K) at time t (FP64-built, stored in the state precision)."""
        v = self._mod.eval("fw_V", self.N, X=self._Xk, t=t).cpu().numpy()
        k = self._mod.eval("fw_K", self.N, P=self._Pk, t=t).cpu().numpy()
        uV = np.exp(-0.5j * self.dt / self.hbar * v)
        uK = np.exp(-1j * self.dt / self.hbar * k)
        return uV, np.conj(uV), uK, np.conj(uK)

    def _vectors(self, times):
        if not (self._v_td or self._k_td):
            key = "static"
            if key not in self._vec_cache:
                self._vec_cache[key] = tuple(self._cvec(a) for a in self._phase_vectors(self.t))
            return self._vec_cache[key] + (0,)
        vs = [self._phase_vectors(t) for t in times]
        return tuple(self._cvec(np.stack([v[q] for v in vs])) for q in range(4)) + (self.N,)

    def _weights(self, times):
        if not self.isEhrenfest:
            return None, None, 0
        def at(t):
            X, P = self._Xk, self._Pk
            wx = np.stack([X, self._mod.eval("fw_dV", self.N, X=X, t=t).cpu().numpy(),
                           self._mod.eval("fw_V", self.N, X=X, t=t).cpu().numpy()])
            g = np.stack([P, self._mod.eval("fw_dK", self.N, P=P, t=t).cpu().numpy(),
                          self._mod.eval("fw_K", self.N, P=P, t=t).cpu().numpy()])
            return wx, np.fft.ifft(g, axis=1)
        if not self._w_td:
            if "w" not in self._vec_cache:
                wx, G = at(self.t)
                self._vec_cache["w"] = (to_device(wx, torch.float64, self.device),
                                        torch.view_as_real(to_device(G, torch.complex128, self.device)).contiguous())
            return self._vec_cache["w"] + (0,)
        pairs = [at(t) for t in times]
        wx = to_device(np.stack([a for a, _ in pairs]), torch.float64, self.device)
        G = torch.view_as_real(to_device(np.stack([b for _, b in pairs]), torch.complex128, self.device)).contiguous()
        return wx, G, 3 * self.N

    def _run(self, n, t0, vectors=None, weights=None):
        """n fused steps after time t0; returns the per-step partial sums (n x M)."""
        times = t0 + self.dt * np.arange(1, n + 1)
        uV, wV, uK, wK, vstep = self._vectors(times) if vectors is None else vectors
        wx, G, wstep = self._weights(times) if weights is None else weights
        Mx = 0 if wx is None else (wx.shape[-2] if wx.dim() >= 2 else 1)
        Mp = 0 if G is None else G.shape[-3]
        M = 4 + 2 * Mx + 2 * Mp
        obs = torch.empty((n, M), dtype=torch.float64, device=self.device)
        d = RhoDesc()
        d.R, d.r_bstride = ptr(self.rho_t), self.N * self.N
        d.uV, d.wV, d.V_step = ptr(uV), ptr(wV), vstep
        d.uK, d.wK, d.K_step = ptr(uK), ptr(wK), vstep
        d.bx, d.bp, d.b_bstride = ptr(self._bx), ptr(self._bp), 0
        d.Mx, d.Mp = Mx, Mp
        d.wx, d.wx_step = ptr(wx), (wstep if wx is not None else 0)
        d.gp, d.gp_step = ptr(G), (2 * wstep if G is not None else 0)  # doubles per step
        d.obs_out, d.dX = ptr(obs), self.dX
        check(self._lib.fw_rho_propagate(self._plan, ctypes.byref(d), n, stream_handle()), "fw_rho_propagate")
        return obs.cpu().numpy()

    def _ehrenfest_from(self, obs):
        tr = obs[:, 0] + 1j * obs[:, 1]
        c = lambda q: obs[:, 4 + 2 * q] + 1j * obs[:, 5 + 2 * q]  # noqa: E731
        self.X_average.extend(np.real(c(0) / tr).tolist())
        self.P_average_RHS.extend((-np.real(c(1) / tr)).tolist())
        self.X_average_RHS.extend(np.real(c(4) / tr).tolist())
        self.P_average.extend(np.real(c(3) / tr).tolist())
        self.hamiltonian_average.extend((np.real(c(5) / tr) + np.real(c(2) / tr)).tolist())

    # -- public API ------------------------------------------------------------
    @property
    def rho(self) -> DeviceArray:
        return DeviceArray(self.rho_t)

    def _normalise_(self):
        tr = complex(self.rho_t.diagonal().sum().item())
        self.rho_t.div_(tr * self.dX)

    def set_rho(self, new_rho):
        """Array (numpy / torch / DeviceArray), F(self, X, X_prime), a C string
        of X, X_prime (i, j), or a float; then normalise by the trace
        (rho_vneumann_cuda_1d.py:301-338)."""
        if isinstance(new_rho, DeviceArray):
            new_rho = new_rho.tensor
        if isinstance(new_rho, (np.ndarray, torch.Tensor)):
            assert tuple(new_rho.shape) == (self.N, self.N), "The grid sizes does not match with the density matrix"
            self.rho_t.copy_(to_device(new_rho, self._ct, self.device))
        elif isinstance(new_rho, FunctionType):
            v = new_rho(self, self.X[:, np.newaxis], self.X[np.newaxis, :])
            self.rho_t.copy_(to_device(np.broadcast_to(v, (self.N, self.N)), self._ct, self.device))
        elif isinstance(new_rho, str):
            mod = cexpr.ExprModule(self.cuda_consts, self.functions, {"fw_init": new_rho})
            N = self.N
            i = np.repeat(np.arange(N), N)
            j = np.tile(np.arange(N), N)
            v = mod.eval("fw_init", N * N, complex_out=True, X=self._Xk[j], X_prime=self._Xk[i], i=i, j=j,
                         indexTotal=j + i * N)
            self.rho_t.copy_(v.view(N, N).to(self._ct))
        elif isinstance(new_rho, float):
            self.rho_t.fill_(new_rho)
        else:
            raise NotImplementedError("new_rho must be either function or numpy.array")
        self._normalise_()
        return self

    def propagate(self, steps=1):
        """t += dt, step, rho /= trace * dX, Ehrenfest (rho_vneumann_cuda_1d.py:355-374)."""
        steps = int(steps)
        per_step = self.isEhrenfest and hasattr(self, "wigner_initial")
        done = 0
        while done < steps:
            n = 1 if per_step else min(self._chunk, steps - done)
            obs = self._run(n, self.t)
            self.t += n * self.dt
            self._last_obs = obs
            if self.isEhrenfest:
                self._ehrenfest_from(obs)
                if per_step:
                    self.wigner_current = self.get_wignerfunction()
                    self.wigner_time.append(self.get_wigner_time(self.wigner_current, self.wigner_initial, self.t))
            done += n
        return self.rho

    def single_step_propagation(self):
        """One step without renormalisation; the reference's cuFFT inverse
        leaves a factor N^2 (rho_vneumann_cuda_1d.py:340-353)."""
        obs = self._run(1, self.t - self.dt, weights=(None, None, 0))
        tr = obs[0, 0] + 1j * obs[0, 1]
        self.rho_t.mul_(tr * self.dX * self.N * self.N)
        return self.rho

    # observables
    def _obs_vector(self, s, p):
        mod = self._observables.get(s)
        if mod is None:
            mod = self._observables[s] = cexpr.ExprModule(self.cuda_consts, self.functions, {"fw_obs": s},
                                                          K=self.K, V=self.V)
        j = np.arange(self.N)
        return mod.eval("fw_obs", self.N, complex_out=True, X=self._Xk, P=self._Pk, t=self.t, j=j, indexTotal=j)

    def _pass(self, R, axis, f0=None, t1=0, f1=None, f2=None, t2=0, f3=None, part=None, ssum=None):
        P = ctypes.POINTER(RhoFactor)
        ref = lambda f: ctypes.byref(f) if f is not None else P()  # noqa: E731
        check(self._lib.fw_rho_pass(self._plan, ptr(R), R.numel(), axis, ref(f0), t1, ref(f1), ref(f2), t2, ref(f3),
                                    ptr(part), ptr(ssum), stream_handle()), "fw_rho_pass")

    def _trace_and_purity(self, R):
        part = torch.empty((self._nparts, 4), dtype=torch.float64, device=self.device)
        self._pass(R, 1, part=part)
        s = part.sum(dim=0).cpu().numpy()
        return complex(s[0], s[1]), float(s[2])

    def get_average(self, observable):
        """Tr[rho O1 O2 ...] dX for a tuple of C strings alternating x- and
        p-operators, None to skip (rho_vneumann_cuda_1d.py:431-472)."""
        self._tmp.copy_(self.rho_t)
        is_x = False
        for s in observable:
            is_x = not is_x
            if not s:
                continue
            vec = self._obs_vector(s, not is_x).to(self._ct)
            if is_x:
                self._pass(self._tmp, 1, f0=_factor(u=vec))
            else:
                self._pass(self._tmp, 1, t1=-1, f1=_factor(1.0 / self.N, u=vec), t2=+1)
        tr, _ = self._trace_and_purity(self._tmp)
        return tr.real * self.dX

    def get_purity(self):
        """sum |rho|^2 dX^2 (rho_vneumann_cuda_1d.py:474-488)."""
        _, p = self._trace_and_purity(self.rho_t)
        return p * self.dX ** 2

    def get_sigma_x_sigma_p(self):
        return np.sqrt((self.get_average(("X * X",)) - self.get_average(("X",)) ** 2)
                       * (self.get_average((None, "P * P")) - self.get_average((None, "P")) ** 2))

    def get_Ehrenfest(self, t):
        if self.isEhrenfest:
            self.X_average.append(self.get_average(("X",)))
            self.X_average_RHS.append(self.get_average((None, self.diff_K)))
            self.P_average.append(self.get_average((None, "P")))
            self.P_average_RHS.append(-self.get_average((self.diff_V,)))
            self.hamiltonian_average.append(self.get_average((None, self.K)) + self.get_average((self.V,)))

    def get_wignerfunction(self):
        """Wigner function of rho by three shears (45 degree rotation) and an FFT
        (rho_vneumann_cuda_1d.py:502-592).  Returns a complex DeviceArray on the
        (P_wigner, X_wigner) grid."""
        N = self.N
        a = np.tan(np.pi / 8.0)
        b = -np.sin(np.pi / 4.0)
        shx = _factor(1.0 / N, shear=(-a, 1, 0, self.dX, self.dP))
        shy = _factor(1.0 / N, shear=(-b, 0, 1, self.dX, self.dP))
        tmp = self._tmp
        tmp.copy_(self.rho_t)
        self._pass(tmp, 1, t1=-1, f1=shx, t2=+1)
        self._pass(tmp, 0, t1=-1, f1=shy, t2=+1)
        self._pass(tmp, 1, t1=-1, f1=shx, t2=+1)
        sg = _factor(sign=True)
        self._pass(tmp, 0, f0=sg, t1=+1, f1=sg)
        ssum = torch.empty((self._nparts, 2), dtype=torch.float64, device=self.device)
        self._pass(tmp, 1, ssum=ssum)
        s = ssum.sum(dim=0).cpu().numpy()
        self._pass(tmp, 1, f0=_factor(1.0 / (complex(s[0], s[1]) * self.wigner_dxdp)))
        return DeviceArray(tmp.clone())

    def get_wigner_time(self, wigner_current, wigner_init, t):
        """int_{H > -Ip} [W - W_init] dxdp with the reference's indicator
        0.5 (1 + signbit(H + Ip)) (rho_vneumann_cuda_1d.py:594-620, 842-857)."""
        mod = self._observables.get("__wigner_time__")
        if mod is None:
            mod = self._observables["__wigner_time__"] = cexpr.ExprModule(
                self.cuda_consts, self.functions,
                {"fw_wt": "0.5 * (1 + int(signbit((%s) + (%s) + Ip)))" % (self.K, self.V)})
        N = self.N
        i = np.repeat(np.arange(N), N)
        j = np.tile(np.arange(N), N)
        ind = mod.eval("fw_wt", N * N, X=self.dX * (j - 0.5 * N) / np.sqrt(2.0),
                       P=self.dP * (i - 0.5 * N) / np.sqrt(2.0), t=t).view(N, N)
        wc = wigner_current.tensor if isinstance(wigner_current, DeviceArray) else torch.as_tensor(wigner_current)
        wi = wigner_init.tensor if isinstance(wigner_init, DeviceArray) else torch.as_tensor(np.asarray(wigner_init))
        wc = wc.to(self.device)
        wc = wc.real if wc.is_complex() else wc
        wi = wi.to(self.device)
        wi = wi.real if wi.is_complex() else wi
        return float((ind * (wc.double() - wi.double())).sum()) * self.wigner_dxdp


class RhoBlochCUDA1D(RhoVNeumannCUDA1D):
    """Gibbs / ground states of rho by the Bloch equation (drop-in for
    rho_bloch_cuda_1d.py:9).  Exponents -dbeta/4 (V + V' - V_min) and
    -dbeta/2 (K + K' - K_min) at t_initial, with K_min = 0 exactly as the
    reference computes it (its fill_K multiplies into a zeroed array, :364)."""

    def __init__(self, **kwargs):
        kwargs = dict(kwargs)
        if "t_initial" not in kwargs:
            kwargs.update(t_initial=0.0)
            print("Warning: Initial time (t_initial) was not specified. So the default value was used t_initial = 0.")
        self.kT = kwargs.pop("kT", 0.0)
        self.dbeta = kwargs.pop("dbeta", 0.01)
        if "dt" not in kwargs:
            kwargs.update(dt=self.dbeta)
        super().__init__(**kwargs)
        ti = float(self.t_initial)
        self._bv = self._mod.eval("fw_V", self.N, X=self._Xk, t=ti).cpu().numpy()
        self._bk = self._mod.eval("fw_K", self.N, P=self._Pk, t=ti).cpu().numpy()
        self.V_min = float(2.0 * self._bv.min())
        self.K_min = 0.0
        self.cuda_consts += "    const double V_min = %.15e;\n" % self.V_min
        self.cuda_consts += "    const double K_min = %.15e;\n" % self.K_min
        self._bw = (to_device(self._bv[None, :], torch.float64, self.device),
                    torch.view_as_real(to_device(np.fft.ifft(self._bk)[None, :], torch.complex128,
                                                 self.device)).contiguous(), 0)
        self._bcache = {}

    def get_V_min(self):
        return self.V_min

    def get_K_min(self):
        return self.K_min

    get_dbeta_num_beta_steps = classmethod(lambda cls, kT, dbeta: _dbeta_steps(kT, dbeta))

    def _bloch_vectors(self, dbeta):
        key = float(dbeta)
        v = self._bcache.get(key)
        if v is None:
            uV = np.exp(-0.25 * dbeta * (self._bv - 0.5 * self.V_min)).astype(complex)
            uK = np.exp(-0.5 * dbeta * (self._bk - 0.5 * self.K_min)).astype(complex)
            v = (self._cvec(uV), self._cvec(uV), self._cvec(uK), self._cvec(uK), 0)
            if len(self._bcache) > 8:
                self._bcache.clear()
            self._bcache[key] = v
        return v

    def _bloch(self, dbeta, n):
        return self._run(n, self.t, vectors=self._bloch_vectors(dbeta), weights=self._bw)

    def bloch_single_step_propagation(self, dbeta):
        """rho_bloch_cuda_1d.py:224-241."""
        self._bloch(float(dbeta), 1)
        return self.rho

    def get_gibbs_state(self, kT=None, dbeta=None, chunk=256):
        """rho_bloch_cuda_1d.py:124-160: delta initial state, stop after the
        first step whose purity is >= 1."""
        dbeta = self.dbeta if dbeta is None else dbeta
        kT = self.kT if kT is None else kT
        dbeta, n = _dbeta_steps(kT, dbeta)
        dbeta = float(dbeta)
        self.set_rho("double(i == j)")
        done = 0
        while done < n:
            m = int(min(chunk, n - done))
            snap = self.rho_t.clone()
            obs = self._bloch(dbeta, m)
            tr2 = obs[:, 0] ** 2 + obs[:, 1] ** 2
            pur = obs[:, 2] / tr2
            bad = np.nonzero(~(pur < 1.0))[0]
            if bad.size:
                k = int(bad[0])
                self.rho_t.copy_(snap)
                self._bloch(dbeta, k + 1)
                kk = done + k
                print("Warning: Gibbs state calculations interupted because purity = %.10f > 1."
                      "Current kT = %.6f" % (self.get_purity(), 1 / (kk * dbeta) if kk else np.inf))
                break
            done += m
        return self.rho

    def get_ground_state(self, dbeta=None, abs_tol_purity=1e-12):
        """rho_bloch_cuda_1d.py:162-222 (purity and energy tests, roll-back)."""
        previous_energy = current_energy = np.inf
        previous_purity = current_purity = 0.0
        dbeta = float(self.dbeta if dbeta is None else dbeta)
        self.set_rho("double(i == j)")
        previous = self.rho_t.clone()
        while current_purity < (1.0 - abs_tol_purity) and dbeta > 1e-12:
            o = self._bloch(dbeta, 1)[0]
            tr = o[0] + 1j * o[1]
            current_purity = float(o[2] / abs(tr) ** 2)
            current_energy = float(np.real((o[4] + 1j * o[5]) / tr) + np.real((o[6] + 1j * o[7]) / tr))
            if current_purity <= 1.0 and current_energy < previous_energy:
                previous_energy, previous_purity = current_energy, current_purity
                previous.copy_(self.rho_t)
                print("Current energy: %.5f; purity: 1 - %.2e; dbeta: %.2e" % (current_energy, 1 - current_purity, dbeta))
            else:
                self.rho_t.copy_(previous)
                dbeta *= 0.5
                current_energy, current_purity = previous_energy, previous_purity
        return self.rho


def _dbeta_steps(kT, dbeta):
    """rho_bloch_cuda_1d.py:99-122."""
    if kT > 0:
        n = 1.0 / (kT * dbeta)
        if round(n) != n:
            n = round(n)
            dbeta = 1.0 / (kT * n)
        return dbeta, int(n)
    return dbeta, np.inf
