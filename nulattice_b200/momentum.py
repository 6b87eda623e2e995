"""Momentum-block CCSD for closed-shell plane-wave inputs.

The plane-wave Hamiltonian of :mod:`nulattice_b200.planewave` (the lattice
contact interaction in the momentum basis, normal-ordered with respect to
closed momentum shells) is what the reference's ``ccsd_solver``
(``CCM/coupled_cluster.py:547-687``) receives as dense blocks; the general
engine then carries t2 as a dense p^2 h^2 tensor (4.4 GB at L=6, A=28) and
evaluates ring terms of p^3 h^3 work.  This module solves the same equations
in the structure those inputs have:

* every hole momentum holds all four spin-isospin states, so f_ph = 0 and
  every T1 term conserves momentum between a particle and a hole, which no
  particle can: t1 stays zero and CCSD reduces to its T2 equation
  (``coupled_cluster.py:476-536`` at t1 = 0);
* t2[a,b,i,j] is non-zero only when k_a + k_b = k_i + k_j = K; it is stored
  in one row-major block per total momentum K of a hole pair, rows
  ``pa*16 + s_a*4 + s_b`` and columns ``pi*16 + s_i*4 + s_j``;
* ``<pq||rs> = V[s_p s_q s_r s_s] delta(K)`` with V independent of the
  momenta, so every diagram reduces to per-block sums and small
  particle-hole intermediates (the kernels in ``csrc/momentum.cu``).

The solver loop is the one of :func:`nulattice_b200.dense.solve` (MP2 start,
Jacobi with mixing, the reference's convergence tests, pulsed DIIS of
``CCM/soa/coupled_cluster.py:479-567``); its iterates equal the general
engine's on the same inputs up to rounding.
"""
from __future__ import annotations

import ctypes
import time

import numpy as np
import torch

from . import _lib
from . import hamiltonian as _ham
from . import planewave as _pw

TILE_ROWS, TILE_COLS = 64, 16


def _madd(L, k1, k2):
    k1, k2 = np.asarray(k1), np.asarray(k2)
    x = (k1 // (L * L) + k2 // (L * L)) % L
    y = ((k1 // L) % L + (k2 // L) % L) % L
    z = (k1 % L + k2 % L) % L
    return (x * L + y) * L + z


def _mneg(L, k):
    k = np.asarray(k)
    return ((-(k // (L * L)) % L) * L + (-((k // L) % L)) % L) * L + (-(k % L)) % L


def contact_tensor(L, n_k, vT1, vS1, w3=0.0):
    """``V[s_p s_q s_r s_s]`` (4^4) of the plane-wave two-body part: the
    contact ``v_loc(vT1, vS1) / L^3`` plus the normal-ordered three-body part,
    an SU(4) contact of strength ``2 n_k w3 / L^3`` (as in
    :func:`planewave.plane_wave_hamiltonian`)."""
    v = _pw._vloc_tensor(vT1, vS1) / L ** 3
    if w3 != 0.0:
        v3 = 2.0 * n_k * w3 / L ** 3
        v = v + _pw._vloc_tensor(v3, v3) / L ** 3
    return v


def fock_blocks(L, n_k, hmom, pmom, vT1, vS1, w3=0.0):
    """Per-momentum 4x4 Fock blocks and E_ref of
    :func:`planewave.plane_wave_hamiltonian` in closed form: kinetic energy
    on the diagonal, the hole trace ``n_k sum_s v2[s_a s s_c s]`` of the
    two-body contact and the three-body ``f_3``; ``E_ref = tr f_hh - 1/2
    sum <kl||kl> + E_3``."""
    v2 = _pw._vloc_tensor(vT1, vS1) / L ** 3
    tr2 = n_k * np.einsum("asbs->ab", v2)
    if w3 != 0.0:
        n_h = 4 * n_k
        e3 = (n_h * (n_h - n_k) * (n_h - 2 * n_k)) / 6.0 * w3 / L ** 6
        f3 = 0.5 * (3 * n_k) * (2 * n_k) * w3 / L ** 6
    else:
        e3 = f3 = 0.0

    def kin(m):
        m = np.asarray(m)
        t = np.zeros(m.shape)
        for c in (m // (L * L), (m // L) % L, m % L):
            t += 2.0 - 2.0 * np.cos(2.0 * np.pi * c / L)
        return t
    eye = np.eye(4)
    fpp = kin(pmom)[:, None, None] * eye + tr2[None] + f3 * eye
    fhh = kin(hmom)[:, None, None] * eye + tr2[None] + f3 * eye
    vt = contact_tensor(L, n_k, vT1, vS1, w3)
    e_ref = float(np.trace(fhh, axis1=1, axis2=2).sum() - 0.5 * n_k ** 2 * np.einsum("stst->", vt) + e3)
    return fpp, fhh, e_ref


class MomentumPlan:
    """Blocked layout of t2 for the closed shells ``holes`` on the L^3
    lattice and the device tables of :c:type:`nlb_pw_problem`."""

    def __init__(self, L, holes):
        holes = np.asarray(holes, dtype=np.int64).reshape(-1, 5)
        self.L = L = int(L)
        n3 = L ** 3
        self.hole, self.part = _ham.ph_split(holes, L)
        hm_states = self.hole // 4
        hmom = np.unique(hm_states)
        if any(np.count_nonzero(hm_states == m) != 4 for m in hmom) or len(self.hole) != 4 * len(hmom):
            raise ValueError("MomentumPlan: every hole momentum needs all four spin-isospin states")
        self.hmom = hmom.astype(np.int64)
        is_h = np.zeros(n3, bool); is_h[hmom] = True
        self.pmom = np.nonzero(~is_h)[0].astype(np.int64)
        self.n_k = len(hmom)
        Ks = np.unique(_madd(L, hmom[:, None], hmom[None, :]).ravel())
        self.Ks = Ks
        pinv = -np.ones(n3, np.int32); pinv[self.pmom] = np.arange(len(self.pmom))
        hinv = -np.ones(n3, np.int32); hinv[self.hmom] = np.arange(len(self.hmom))
        kblk = -np.ones(n3, np.int32); kblk[Ks] = np.arange(len(Ks))
        ppos = -np.ones((len(Ks), n3), np.int32)
        hpos = -np.ones((len(Ks), n3), np.int32)
        pm_list, hm_list, nr, nc, pm0, hm0 = [], [], [], [], [], []
        for q, K in enumerate(Ks):
            partner_p = _madd(L, K, _mneg(L, self.pmom))
            pm = self.pmom[~is_h[partner_p]]
            partner_h = _madd(L, K, _mneg(L, self.hmom))
            hmk = self.hmom[is_h[partner_h]]
            ppos[q, pm] = np.arange(len(pm)); hpos[q, hmk] = np.arange(len(hmk))
            pm0.append(sum(len(x) for x in pm_list)); hm0.append(sum(len(x) for x in hm_list))
            pm_list.append(pinv[pm]); hm_list.append(hinv[hmk])
            nr.append(16 * len(pm)); nc.append(16 * len(hmk))
        self.nr, self.nc = np.array(nr, np.int64), np.array(nc, np.int64)
        self.blk_off = np.concatenate([[0], np.cumsum(self.nr * self.nc)]).astype(np.int64)
        self.m_off = np.concatenate([[0], np.cumsum(16 * self.nc)]).astype(np.int64)
        self.w_off = np.concatenate([[0], np.cumsum(self.nc * self.nc)]).astype(np.int64)
        self.row_off = np.concatenate([[0], np.cumsum(self.nr)]).astype(np.int64)
        self.n_t2 = int(self.blk_off[-1])
        self.pm_list = np.concatenate(pm_list).astype(np.int32)
        self.hm_list = np.concatenate(hm_list).astype(np.int32)
        self.pm0, self.hm0 = np.array(pm0, np.int32), np.array(hm0, np.int32)
        self.ppos, self.hpos, self.kblk, self.pinv, self.hinv = ppos, hpos, kblk, pinv, hinv
        tiles = [(q, r0, c0) for q in range(len(Ks)) for r0 in range(0, int(self.nr[q]), TILE_ROWS)
                 for c0 in range(0, int(self.nc[q]), TILE_COLS)]
        self.tiles = np.array(tiles, np.int32).reshape(-1, 3)
        self.p, self.h = len(self.part), len(self.hole)

    # -- dense conversion (tests, small cases) ----------------------------
    def _index_grid(self):
        """Generic (a, b, i, j) of every blocked amplitude, in block order."""
        L = self.L
        pidx = -np.ones(4 * L ** 3, np.int64); pidx[self.part] = np.arange(self.p)
        hidx = -np.ones(4 * L ** 3, np.int64); hidx[self.hole] = np.arange(self.h)
        out = []
        for q, K in enumerate(self.Ks):
            pm = self.pmom[self.pm_list[self.pm0[q]:self.pm0[q] + self.nr[q] // 16]]
            hm = self.hmom[self.hm_list[self.hm0[q]:self.hm0[q] + self.nc[q] // 16]]
            ma = np.repeat(pm, 16); s = np.tile(np.arange(16), len(pm))
            mb = _madd(L, K, _mneg(L, ma))
            a = pidx[ma * 4 + s // 4]; b = pidx[mb * 4 + s % 4]
            mi = np.repeat(hm, 16); u = np.tile(np.arange(16), len(hm))
            mj = _madd(L, K, _mneg(L, mi))
            i = hidx[mi * 4 + u // 4]; j = hidx[mj * 4 + u % 4]
            out.append((np.repeat(a, len(i)), np.repeat(b, len(i)), np.tile(i, len(a)), np.tile(j, len(a))))
        return tuple(np.concatenate([o[k] for o in out]) for k in range(4))

    def to_dense(self, t2):
        """Dense (p, p, h, h) array in the generic state order of
        :func:`hamiltonian.ph_split` (small cases only)."""
        t = np.asarray(t2.detach().cpu() if isinstance(t2, torch.Tensor) else t2, dtype=np.float64)
        out = np.zeros((self.p, self.p, self.h, self.h))
        out[self._index_grid()] = t
        return out

    def from_dense(self, t2):
        """Blocked amplitudes of a dense (p, p, h, h) array."""
        return np.asarray(t2, dtype=np.float64)[self._index_grid()]

    # -- device problem ----------------------------------------------------
    def problem(self, V, fpp, fhh, device):
        """The :c:type:`nlb_pw_problem` with its tables on ``device``."""
        dev = torch.device(device)
        i32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int32), device=dev)  # noqa: E731
        i64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.int64), device=dev)  # noqa: E731
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)  # noqa: E731
        keep = dict(blk_off=i64(self.blk_off), m_off=i64(self.m_off), w_off=i64(self.w_off),
                    row_off=i64(self.row_off), blk_nr=i32(self.nr), blk_nc=i32(self.nc), blk_K=i32(self.Ks),
                    blk_pm0=i32(self.pm0), blk_hm0=i32(self.hm0), pm_list=i32(self.pm_list),
                    hm_list=i32(self.hm_list), ppos=i32(self.ppos), hpos=i32(self.hpos), kblk=i32(self.kblk),
                    pmom=i32(self.pmom), hmom=i32(self.hmom), pinv=i32(self.pinv), hinv=i32(self.hinv),
                    tiles=i32(self.tiles), V=f64(np.asarray(V).reshape(256)), fpp=f64(np.asarray(fpp).reshape(-1)),
                    fhh=f64(np.asarray(fhh).reshape(-1)))
        P = _lib.PwProblem()
        P.L, P.n_blocks, P.n_pmom, P.n_hmom = self.L, len(self.Ks), len(self.pmom), len(self.hmom)
        P.n_t2, P.n_m, P.n_w, P.n_rows = self.n_t2, int(self.m_off[-1]), int(self.w_off[-1]), int(self.row_off[-1])
        P.n_tiles = len(self.tiles)
        for k, t in keep.items():
            setattr(P, k, t.data_ptr())
        return P, keep


class MomentumEngine:
    """Device tables, intermediates and the entry points (``nlb_pw_init`` /
    ``nlb_pw_energy`` / ``nlb_pw_step``, or their ``_f32`` twins) of one
    problem.  ``dtype`` is the type of the amplitudes and intermediates
    (torch.float64, or torch.float32 for the first phase of a mixed solve);
    ``tables``: another engine of the same problem whose device tables are
    shared."""

    def __init__(self, plan, V, fpp, fhh, device=None, dtype=torch.float64, tables=None):
        self.plan = plan
        self.dev = torch.device(device if device is not None else "cuda")
        self.L = _lib.lib()
        if tables is not None:
            self.P, self._keep = tables.P, tables._keep
        else:
            self.P, self._keep = plan.problem(V, fpp, fhh, self.dev)
        self.dtype = dtype
        self.f32 = dtype == torch.float32
        self.stream = torch.cuda.current_stream(self.dev)
        self.sp = ctypes.c_void_p(self.stream.cuda_stream)
        P = self.P
        z = lambda k: torch.zeros(k, dtype=dtype, device=self.dev)  # noqa: E731
        nph = 4 * P.n_pmom * 4 * P.n_hmom * 16
        self.bufs = dict(M=z(P.n_m), W=z(P.n_w), Y=z(4 * P.n_rows), Xpp=z(16 * P.n_pmom), Xhh=z(16 * P.n_hmom),
                         R=z(nph), U=z(nph), G=z(nph), H=z(plan.n_t2),
                         energy=torch.zeros(1, dtype=torch.float64, device=self.dev))
        self.S = _lib.PwState(**{k: v.data_ptr() for k, v in self.bufs.items()})
        self.launches = 0

    def zeros(self):
        return torch.zeros(self.plan.n_t2, dtype=self.dtype, device=self.dev)

    def init(self, t2, delta=0.0):
        """MP2 start into ``t2`` (formed in FP64)."""
        x = t2 if not self.f32 else torch.zeros(self.plan.n_t2, dtype=torch.float64, device=self.dev)
        _lib.check(self.L.nlb_pw_init(ctypes.byref(self.P), x.data_ptr(), float(delta), self.sp), "pw init")
        if self.f32:
            t2.copy_(x)
        self.launches += 1

    def energy(self, t2):
        """Energy of ``t2`` (device scalar, FP64); also leaves M of ``t2`` for the next step."""
        fn = self.L.nlb_pw_energy_f32 if self.f32 else self.L.nlb_pw_energy
        _lib.check(fn(ctypes.byref(self.P), t2.data_ptr(), ctypes.byref(self.S), self.sp), "pw energy")
        self.launches += 3
        return self.bufs["energy"]

    def step(self, t2, out, err=None, mixing=0.5):
        """One Jacobi step with mixing from ``t2`` (M of ``t2`` current) into ``out``."""
        fn = self.L.nlb_pw_step_f32 if self.f32 else self.L.nlb_pw_step
        _lib.check(fn(ctypes.byref(self.P), t2.data_ptr(), out.data_ptr(),
                      err.data_ptr() if err is not None else None, float(mixing), ctypes.byref(self.S), self.sp),
                   "pw step")
        self.launches += 6


def jacobi_gap(eng, t2):
    """Largest change of one unmixed Jacobi step at ``t2``: zero at the CCSD
    fixed point (the reference's residual test)."""
    out = eng.zeros()
    eng.energy(t2)
    eng.step(t2, out, mixing=0.0)
    return float((out - t2).abs().max().item())


def _iterate(eng, xs, cur, eps, maxSteps, max_diis, mixing, criterion, verbose, step0=0):
    """The solver loop on engine ``eng`` from the amplitudes ``xs[cur]``.
    Returns (E, cur, status, steps).

    The energy of each step comes back through a page-locked slot and an
    event, and the next step is queued before that energy is read, so the
    device does not wait for the host's convergence test.  Only a step after
    which a DIIS extrapolation is due waits for its test first (the
    extrapolation rewrites the amplitudes in place).  A step queued after
    the converged one writes the buffer of the step before, so the converged
    amplitudes stay untouched; the steps, and so the results, are the same
    as with a test after every step."""
    L, sp = eng.L, eng.sp
    n = eng.plan.n_t2
    use_diis = criterion == "soa" and max_diis > 0
    if use_diis:
        # every error / history row is written before an extrapolation reads it
        err = torch.empty((max_diis, n), dtype=eng.dtype, device=eng.dev)
        hist = torch.empty((max_diis, n), dtype=eng.dtype, device=eng.dev)
        work = torch.zeros(_lib.NLB_DENSE_WORK_DOUBLES, dtype=torch.float64, device=eng.dev)
        diis = L.nlb_vec_diis_f32 if eng.f32 else L.nlb_vec_diis_f64
    nerr = 0
    if getattr(eng, "_host_e", None) is None:   # page-locked energy slots, kept on the engine
        eng._host_e = torch.zeros(2, dtype=torch.float64, pin_memory=True)
        eng._events = [torch.cuda.Event(), torch.cuda.Event()]
    host_e, events = eng._host_e, eng._events

    def launch(k, src, e_slot):
        """Step k from xs[src] into xs[src ^ 1] (DIIS error into err[e_slot]),
        its energy, and the energy's copy into host slot k % 2."""
        eng.step(xs[src], xs[src ^ 1], err[e_slot] if use_diis else None, mixing)
        eng.energy(xs[src ^ 1])
        with torch.cuda.stream(eng.stream):
            host_e[k % 2:k % 2 + 1].copy_(eng.bufs["energy"], non_blocking=True)
            events[k % 2].record(eng.stream)

    prev = float(eng.energy(xs[cur]).item())
    if verbose and step0 == 0:
        print(f"Step 0: {prev}")
    status, e, it = "max_iter", prev, 0
    if maxSteps >= 1:
        launch(1, cur, nerr)
    for it in range(1, maxSteps + 1):
        # step `it` (xs[cur] -> xs[cur ^ 1]) is queued; queue step it + 1
        # unless a DIIS extrapolation would come between them
        ahead = it < maxSteps and (not use_diis or nerr + 1 < max_diis)
        if ahead:
            if use_diis:
                hist[nerr].copy_(xs[cur ^ 1])
            launch(it + 1, cur ^ 1, nerr + 1 if use_diis else 0)
        events[it % 2].synchronize()
        e = float(host_e[it % 2])
        cur ^= 1
        if verbose:
            print(f"Step {step0 + it}: {e}", "difference =", abs(e - prev) / abs(e) if e != 0 else float("inf"))
        if criterion == "soa":
            done = abs(e - prev) / max(1.0, abs(e)) < eps
        else:
            done = (e == 0 and prev == 0) or (e != 0 and abs(e - prev) / abs(e) < eps)
        if done:
            status = "converged"
            break
        if use_diis:
            if not ahead:
                hist[nerr].copy_(xs[cur])
            nerr += 1
            if nerr == max_diis:
                _lib.check(diis(err.data_ptr(), hist.data_ptr(), n, max_diis, work.data_ptr(), xs[cur].data_ptr(),
                                sp), "pw diis")
                eng.launches += 4
                eng.energy(xs[cur])    # M of the extrapolated amplitudes for the next step
                nerr = 0
        if abs(e) > 1e10 or e != e:
            status = "diverged"
            break
        prev = e
        if not ahead and it < maxSteps:
            launch(it + 1, cur, nerr)
    return e, cur, status, it


def solve(plan, V, fpp, fhh, eps=1e-8, maxSteps=1000, max_diis=10, delta=0.0, mixing=0.5, verbose=False,
          criterion="soa", device=None, info=None, engine=None, precision="fp64", mixed_eps=None):
    """The solver loop of :func:`nulattice_b200.dense.solve` on the blocked
    amplitudes.  Returns ``(E_corr, t2)``, t2 blocked on the device (FP64).

    ``precision="mixed"``: FP32 amplitudes and intermediates (FP64 energy,
    DIIS algebra in FP64) until the energy test passes at ``mixed_eps``
    (default ``max(eps, 1e-7)``), then FP64 from the converted amplitudes to
    ``eps``.  ``engine``: an FP64 engine of the problem (reused)."""
    info = {} if info is None else info
    t0 = time.perf_counter()
    eng = engine if engine is not None else MomentumEngine(plan, V, fpp, fhh, device)
    xs = [eng.zeros(), eng.zeros()]
    cur, done_steps = 0, 0
    launches0 = eng.launches
    if precision == "mixed":
        e32 = getattr(eng, "_f32_twin", None)
        if e32 is None:
            e32 = eng._f32_twin = MomentumEngine(plan, V, fpp, fhh, eng.dev, dtype=torch.float32, tables=eng)
        l32 = e32.launches
        ys = [e32.zeros(), e32.zeros()]
        e32.init(ys[0], delta)
        me = float(mixed_eps) if mixed_eps is not None else max(float(eps), 1e-7)
        e, c32, status, done_steps = _iterate(e32, ys, 0, me, maxSteps, max_diis, mixing, criterion, verbose)
        info.update(mixed_iters=done_steps, mixed_energy=e, mixed_status=status)
        launches0 -= e32.launches - l32
        xs[0].copy_(ys[c32])
        if status == "converged" and maxSteps - done_steps > 0:
            e, cur, status, it = _iterate(eng, xs, 0, eps, maxSteps - done_steps, max_diis, mixing, criterion,
                                          verbose, step0=done_steps)
            done_steps += it
    else:
        eng.init(xs[0], delta)
        e, cur, status, done_steps = _iterate(eng, xs, 0, eps, maxSteps, max_diis, mixing, criterion, verbose)
    eng.stream.synchronize()
    if status == "max_iter":
        print("Max iterations reached.")
    info.update(status=status, iterations=done_steps, t_iterate=time.perf_counter() - t0,
                launches=eng.launches - launches0, engine="momentum", n_t2=plan.n_t2, blocks=len(plan.Ks),
                precision=precision)
    return e, xs[cur]


def ccsd_plane_wave(L, holes, vT1, vS1, w3=0.0, eps=1e-8, maxSteps=1000, max_diis=10, delta=0.0, mixing=0.5,
                    verbose=False, criterion="soa", device=None, info=None, precision="fp64", mixed_eps=None):
    """CCSD of the closed-shell plane-wave Hamiltonian
    :func:`planewave.plane_wave_hamiltonian` ``(L, holes, vT1, vS1, w3)`` on
    the momentum blocks.  Returns ``(E_corr, E_ref, t2, plan)``: t2 blocked
    on the device (``plan.to_dense`` gives the reference's layout)."""
    info = {} if info is None else info
    t0 = time.perf_counter()
    plan = MomentumPlan(L, holes)
    V = contact_tensor(L, plan.n_k, vT1, vS1, w3)
    fpp, fhh, e_ref = fock_blocks(L, plan.n_k, plan.hmom, plan.pmom, vT1, vS1, w3)
    info["t_plan"] = time.perf_counter() - t0
    e, t2 = solve(plan, V, fpp, fhh, eps=eps, maxSteps=maxSteps, max_diis=max_diis, delta=delta, mixing=mixing,
                  verbose=verbose, criterion=criterion, device=device, info=info, precision=precision,
                  mixed_eps=mixed_eps)
    return e, e_ref, t2, plan
