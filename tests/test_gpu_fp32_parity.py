"""The FP32 kernels against Oracle32, the oracle built with float step arithmetic, one step at a time.

Both compute the geometry in double and round it once to float, step the state, gradients,
limiter and fluxes in float, sum each cell's residual with a compensated two-sum, and keep the
dt minimum and the residual norm in double.  They differ in one respect: the GPU's FP32 path
uses the hardware's approximate reciprocal, quotient and square root (__fdividef, rsqrtf, each
within a few float ulps), the oracle IEEE float.

The oracle restarts every step from the GPU's state, so each comparison measures the
arithmetic of one step: differences cannot build up through the limiter's switches.

Tolerance, in float ulps (EPS32 = 2^-23, the spacing of floats in [1, 2)): after each step the
relative L-infinity distance per conserved variable (max |a-b| / max |b|, ghost cells included)
is at most STATE_ULPS * EPS32; the step's dt at most DT_ULPS * EPS32 relative; the L2 density
residual at most RES_ULPS * EPS32 relative.
"""
import numpy as np
import pytest

import cfd_optimisations_b200 as H
from cfd_optimisations_b200.arena import Arena
import oracle as O

pytestmark = pytest.mark.gpu

EPS32 = 2.0 ** -23
STATE_ULPS = 4
DT_ULPS = 4
RES_ULPS = 4

STEPS = 30


def _oracle32(mesh, bcmap, qbc, q, limiter, K):
    o = O.Oracle32(mesh.arrays())
    o.gather_bcs(bcmap, qbc)
    o.initialise(q)
    o.set_limiter(O.VENKAT if limiter == H.LIMITER_VENKAT else O.BJ, K)
    return o


def _check_step(U_gpu, st, o, U_start, mode, cfl, where):
    o.set_U(U_start)
    dt_o, res_o = o.step(mode, cfl)
    err = O.rel_linf(U_gpu, o.U())
    assert np.all(err <= STATE_ULPS * EPS32), (where, err / EPS32)
    if mode != H.FIXED_DT:
        assert abs(st["dt"] - dt_o) <= DT_ULPS * EPS32 * dt_o, (where, st["dt"], dt_o)
    assert abs(st["res_l2"] - res_o) <= RES_ULPS * EPS32 * res_o, (where, st["res_l2"], res_o)


@pytest.mark.parametrize("kernel", [H.KERNEL_TILED, H.KERNEL_CELL])
@pytest.mark.parametrize("limiter,K", [(H.LIMITER_BJ, 0.0), (H.LIMITER_VENKAT, 5.0)])
@pytest.mark.parametrize("mode,cfl", [(H.GLOBAL_CFL, 0.5), (H.LOCAL_CFL, 0.8)])
def test_fp32_single_mesh_steps_match_oracle32(kernel, limiter, K, mode, cfl):
    m = H.Mesh.wedge(161, 81, theta_deg=15.0, seed=1234, numbering=H.NUMBER_RANDOM)
    bcmap, qbc, q = H.wedge_case(2.5)
    s = H.Solver(m, limiter=limiter, venkat_K=K, precision=H.FP32, kernel=kernel)
    s.gather_bcs(bcmap, qbc)
    s.initialise(q)
    o = _oracle32(m, bcmap, qbc, q, limiter, K)
    assert np.all(O.rel_linf(s.U(), o.U()) <= EPS32)
    for i in range(STEPS):
        U0 = s.U()
        st = s.step(1, mode, cfl)
        _check_step(s.U(), st, o, U0, mode, cfl, i)


@pytest.mark.parametrize("limiter,K", [(H.LIMITER_BJ, 0.0), (H.LIMITER_VENKAT, 5.0)])
def test_fp32_arena_steps_match_oracle32(limiter, K):
    """Three wedges of different sizes and Mach numbers in one FP32 arena (tiled kernels in
    arena mode), each compared with its own Oracle32 every step."""
    cases = [(H.Mesh.wedge(121, 61, theta_deg=12.0, seed=2), 3.1), (H.Mesh.wedge(81, 41, theta_deg=5.0, seed=3), 2.4),
             (H.Mesh.wedge(61, 31, theta_deg=15.0, seed=4), 1.9)]
    a = Arena(1 << 27, precision=H.FP32, limiter=limiter, venkat_K=K)
    inst = []
    for m, M in cases:
        bcmap, qbc, q = H.wedge_case(M)
        k = a.admit(m, bcmap, qbc, q, 0.5)
        o = _oracle32(m, bcmap, qbc, q, limiter, K)
        assert np.all(O.rel_linf(a.fetch(k), o.U()) <= EPS32)
        inst.append((k, o))
    for i in range(STEPS):
        U0 = [a.fetch(k) for k, _ in inst]
        a.step(1)
        stats = a.poll()
        for (k, o), u0 in zip(inst, U0):
            _check_step(a.fetch(k), stats[k], o, u0, H.GLOBAL_CFL, 0.5, (k, i))
