"""Batched and served execution (pxp_batch_*, paxpro_b200.serving).

The requirement: every result is the same alone and in the mix.  Each job
runs on its own CTA (2-D) or its own stream (3-D) with the same kernels and
inputs as a solver stepped alone, so the check is bitwise equality of the
exit intensities, in FP64 and in FP32 served mode."""
import numpy as np
import pytest

from paxpro_b200 import workloads as wl

pytestmark = pytest.mark.gpu


def _jobs():
    from paxpro_b200 import serving as sv
    rng = np.random.default_rng(7)
    jobs = []
    for i in range(14):
        kind = "fft2d" if i % 3 else "cn"
        j = sv.draw_2d(rng, kind, i)
        j.n = [256, 512, 1024, 2048, 4096, 8192, 256][i % 7]
        if kind == "cn":
            j.n = min(j.n, 4096)
        j.nsteps = int(rng.integers(20, 120))
        jobs.append(j)
    for i in range(3):
        j = sv.draw_3d(rng, 100 + i, sizes=(256, 512))
        j.nsteps = int(rng.integers(5, 15))
        jobs.append(j)
    return jobs


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_results_equal_alone(precision):
    from paxpro_b200 import serving as sv
    jobs = _jobs()
    alone = sv.run_plain(jobs, precision=precision)
    # rounds of 17 steps so that jobs enter and leave mid-batch
    mixed = sv.run_batched(jobs, precision=precision, max_steps=17)
    for i in range(len(jobs)):
        assert np.array_equal(alone.intensities[i], mixed.intensities[i]), (i, jobs[i].kind, jobs[i].n)


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_sizes_other_than_powers_of_two_equal_alone(precision):
    """Batch groups on padded and Bluestein kernels (CrankNicholson at 300
    and 600 rows on the step-invariant path padded to 512 and 1024;
    FFTSolver2D at 1000 and 3000 points by Bluestein's transform) and the
    largest lines (FFTSolver2D at 16384 points: a two-CTA cluster in FP64),
    entering and leaving mid-batch: every exit intensity equal bit for bit
    to the solver stepped alone."""
    from paxpro_b200 import serving as sv
    rng = np.random.default_rng(11)
    jobs = []
    for i, (kind, n) in enumerate([("cn", 300), ("cn", 300), ("cn", 600), ("fft2d", 1000),
                                   ("fft2d", 3000), ("fft2d", 16384), ("fft2d", 1000)]):
        j = sv.draw_2d(rng, kind, i)
        j.n = n
        j.nsteps = int(rng.integers(20, 90))
        jobs.append(j)
    alone = sv.run_plain(jobs, precision=precision)
    mixed = sv.run_batched(jobs, precision=precision, max_steps=13)
    for i in range(len(jobs)):
        assert np.array_equal(alone.intensities[i], mixed.intensities[i]), (i, jobs[i].kind, jobs[i].n)


def test_batch_budget_refuses_and_releases():
    import paxpro_b200 as pxp
    from paxpro_b200 import serving as sv
    rng = np.random.default_rng(1)
    j = sv.draw_2d(rng, "fft2d", 0)
    j.n, j.nsteps = 2048, 10
    s1 = sv.make_solver(j, 1)
    s2 = sv.make_solver(j, 1)
    b = pxp.Batch(0, hbm_budget_bytes=s1.device_bytes() + s2.device_bytes() // 2)
    assert b.admit(s1, j.nsteps)
    assert not b.admit(s2, j.nsteps)  # over budget: not admitted
    b.round(100)
    assert [x._h.value for x in b.collect()] == [s1._h.value]
    assert b.admit(s2, j.nsteps)      # memory released by the finished job
    b.round(100)
    assert len(b.collect()) == 1
    b.close()
    s1.close()
    s2.close()


def test_serving_results_equal_alone():
    from paxpro_b200 import serving as sv
    jobs = sv.served_jobs(rate=400.0, duration=0.05, seed=9)
    for j in jobs:
        j.nsteps = min(j.nsteps, 150)
        if j.kind == "fft3d":
            j.n = min(j.n, 512)
            j.nsteps = min(j.nsteps, 20)
    served = {}
    res = sv.serve(jobs, precision=1, round_steps=40, results=served, realtime=False)
    assert len(res.latencies) == len(jobs) and res.max_active > 1
    alone = sv.run_plain(jobs, precision=1)
    for i in range(len(jobs)):
        assert np.array_equal(served[i], alone.intensities[i]), (i, jobs[i].kind)
