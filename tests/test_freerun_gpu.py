"""Free-run parity on the chaotic infinite-plane workload (N = 1024, RK4, dt = 1e-3, 100 steps).

A 1-ulp change of one coordinate grows to O(1) within ~40 steps of this state, so no two FP64
implementations can agree on the final positions. The criterion is the reference's own
sensitivity to rounding: the GPU trajectory may not drift from the reference CPU trajectory
faster than the reference drifts from itself (a) when every coordinate of the initial state is
moved by one ulp (seeded random directions) and (b) when it sums the sources of every
evaluation in reverse order (an equally valid FP64 evaluation that rounds differently at every
step, which is what a different implementation does). The envelope of the two is the bound, with
a factor 10 for where the first differences land. Measured on this state (reference CPU):
(a) 9.6e-11 / 1.1e-8 after 5 / 10 steps, (b) 2.4e-10 / 2.8e-7; moving one coordinate only
understates both, because the fastest vortices (tight pairs, speeds ~1e4) amplify a rounding
difference the most. Invariants that the
dynamics conserve exactly (circulation, linear impulse) must be conserved as tightly as the
reference conserves them; the Hamiltonian and angular impulse drifts may not exceed the envelope
of the reference's own runs."""
import numpy as np
import pytest

import pointvortex_b200 as pv
from oracle.pyoracle import Geometry
from pointvortex_b200 import ics

pytestmark = pytest.mark.gpu


def test_free_run_divergence_no_worse_than_reference_self_divergence(reference):
    x, y, g = ics.workload_state("infinite_rk4_n1024")
    geo = Geometry("infinite")
    checkpoints = (5, 10, 20, 40, 100)

    def cpu_run_g(x0, y0, g0):
        st = reference.stepper(geo, x0.size)
        cx, cy, out = x0.copy(), y0.copy(), {}
        for k in range(1, 101):
            cx, cy = st.rk4_step(cx, cy, g0, 1e-3)
            if k in checkpoints:
                out[k] = (cx.copy(), cy.copy())
        return out

    def cpu_run(x0, y0):
        return cpu_run_g(x0, y0, g)

    ref = cpu_run(x, y)
    rng = np.random.default_rng(1)
    xp = np.nextafter(x, x + (2 * rng.integers(0, 2, x.size) - 1) * np.inf)
    yp = np.nextafter(y, y + (2 * rng.integers(0, 2, y.size) - 1) * np.inf)
    perturbed = cpu_run(xp, yp)
    rev = np.arange(x.size)[::-1]
    back = np.argsort(rev)
    reordered = {c: (px[back], py[back])
                 for c, (px, py) in cpu_run_g(x[rev], y[rev], g[rev]).items()}

    k = pv.InfinitePlaneKernel(0.0)
    k.uploadDeviceState(pv.VortexSystem(x, y, g))
    gpu, done = {}, 0
    for c in checkpoints:
        k.rk4Advance(1e-3, c - done)
        done = c
        s = pv.VortexSystem(x.copy(), y.copy(), g)
        k.downloadDeviceState(s)
        gpu[c] = (s.x, s.y)

    for c in checkpoints:
        d_gpu = np.max(np.hypot(gpu[c][0] - ref[c][0], gpu[c][1] - ref[c][1]))
        d_ulp = np.max(np.hypot(perturbed[c][0] - ref[c][0], perturbed[c][1] - ref[c][1]))
        d_rev = np.max(np.hypot(reordered[c][0] - ref[c][0], reordered[c][1] - ref[c][1]))
        print(f"step {c}: gpu-vs-cpu {d_gpu:.3e}; reference vs itself: 1-ulp state {d_ulp:.3e}, "
              f"reversed summation {d_rev:.3e}")
        assert d_gpu <= 10.0 * max(d_ulp, d_rev, 1e-15), (c, d_gpu, d_ulp, d_rev)

    inv0 = reference.invariants(geo, x, y, g)
    inv_cpu = reference.invariants(geo, ref[100][0], ref[100][1], g)
    inv_gpu = k.stateInvariants()
    gpu_arr = np.array([inv_gpu.circulation, inv_gpu.linearImpulseX, inv_gpu.linearImpulseY,
                        inv_gpu.angularImpulse, inv_gpu.hamiltonian])
    drift_cpu = np.abs(inv_cpu - inv0)
    drift_gpu = np.abs(gpu_arr - inv0)
    # the reference's own runs from the 1-ulp state and with reversed summation
    drift_ulp = np.abs(reference.invariants(geo, *perturbed[100], g)
                       - reference.invariants(geo, xp, yp, g))
    drift_rev = np.abs(reference.invariants(geo, *reordered[100], g) - inv0)
    envelope = np.max([drift_cpu, drift_ulp, drift_rev], axis=0)
    print("drift cpu", drift_cpu, "1-ulp", drift_ulp, "reversed", drift_rev, "gpu", drift_gpu)
    assert drift_gpu[0] <= 1e-12
    assert drift_gpu[1] <= max(10 * drift_cpu[1], 1e-12) and drift_gpu[2] <= max(10 * drift_cpu[2], 1e-12)
    # The Hamiltonian and the angular impulse are conserved by the flow but not by RK4 at this
    # step: a few tight pairs are under-resolved, and how much H and L drift depends on the
    # chaotic details. Over the reference's own runs from this state (1-ulp perturbations, reversed
    # summation) |dH| spans 14.1-17.8 and |dL| 0.003-0.024. The GPU's drift may not be larger
    # than the envelope of the three reference runs made here, with a factor 1.5 for H and 3 for
    # L (whose spread between runs is relatively wider).
    assert drift_gpu[4] <= 1.5 * envelope[4], (drift_gpu[4], envelope[4])
    assert drift_gpu[3] <= 3.0 * envelope[3], (drift_gpu[3], envelope[3])
