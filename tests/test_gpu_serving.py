"""Form (c): the serving loop.  Each job's images are the same served alone,
served in a mix of engines and sizes with shots joining between ticks, and
computed by the one-shot path; a failing job fails alone."""

from __future__ import annotations

import numpy as np
import pytest

from test_gpu_batch import _inputs

pytestmark = pytest.mark.gpu

CASES = ("mig_acoustic_zerolag", "mig_elastic_pp_divcurl", "mig_visco_comp", "mig_acoustic_excitation")


def _job(case: str, n_shots: int = 3):
    from ertm_b200 import RTMImager
    from ertm_b200.serving import ServeJob
    fx, model, shots, imaging, solver, q = _inputs(case)
    imager = RTMImager(imaging, solver, q)
    modes = ("pp", "ps") if fx["meta"]["engine"] == "elastic" else ("pp",)
    return ServeJob(shots=shots[:n_shots], model=model, imager=imager, modes=modes, name=case)


def _plain(job):
    from ertm_b200.stacking import stack_images
    per = [job.imager.migrate_modes(s, job.model, modes=job.modes) for s in job.shots]
    return [stack_images([p[k] for p in per]).image for k in range(len(job.modes))]


def _serve(jobs, **kw):
    from ertm_b200.serving import RTMServer
    with RTMServer(**kw) as srv:
        futs = [srv.submit(j) for j in jobs]
        out = [f.result(timeout=600) for f in futs]
    return out, srv.summary()


def test_served_alone_equals_one_shot_path():
    for case in CASES:
        job = _job(case)
        (res,), summary = _serve([job])
        for img, ref in zip(res.images, _plain(job)):
            assert np.array_equal(img.image, ref), case
        assert summary["jobs_done"] == 1 and summary["shots_done"] == len(job.shots)


def test_mixed_stream_equals_alone():
    """Four jobs of three engines; at most four shots at a time and short polls,
    so shots of later jobs join while earlier ones are mid-run."""
    jobs = [_job(c) for c in CASES]
    alone = [_serve([j])[0][0] for j in jobs]
    mixed, summary = _serve(jobs, max_shots=4, ticks_per_poll=7)
    for a, m in zip(alone, mixed):
        for x, y in zip(a.images, m.images):
            assert np.array_equal(x.image, y.image), a.name
    assert summary["peak_active"] == 4
    assert summary["shot_latency_p99_s"] >= summary["shot_latency_p50_s"] > 0
    assert summary["jobs_done"] == len(jobs)


def test_failed_job_fails_alone():
    """A mode the engine cannot image, and a failure planted on the host at a
    shot's completion: those two jobs raise, the others are unchanged."""
    from ertm_b200.exceptions import ImagingError
    good = _job("mig_acoustic_zerolag")
    bad_mode = _job("mig_acoustic_norm_rn")
    bad_mode.modes = ("ps",)
    planted = _job("mig_elastic_pp_divcurl")

    def hook(stage, job_id, shot):
        if stage == "finish" and job_id == 2 and shot == 1:
            raise RuntimeError("planted host-side failure")

    from ertm_b200.serving import RTMServer
    with RTMServer(max_shots=3, ticks_per_poll=5, fault_hook=hook) as srv:
        f_good, f_bad, f_planted, f_good2 = (srv.submit(good), srv.submit(bad_mode), srv.submit(planted),
                                             srv.submit(good))
        with pytest.raises(ImagingError):
            f_bad.result(timeout=600)
        with pytest.raises(RuntimeError, match="planted"):
            f_planted.result(timeout=600)
        r1, r2 = f_good.result(timeout=600), f_good2.result(timeout=600)
    ref = _plain(good)
    assert np.array_equal(r1.images[0].image, ref[0]) and np.array_equal(r2.images[0].image, ref[0])
    assert srv.summary()["jobs_failed"] == 2


def test_budget_too_small_for_a_shot():
    from ertm_b200.exceptions import ImagingError
    (job,) = [_job("mig_acoustic_zerolag", 1)]
    from ertm_b200.serving import RTMServer
    with RTMServer(memory_budget=1024) as srv:
        f = srv.submit(job)
        with pytest.raises(ImagingError, match="budget"):
            f.result(timeout=120)


def test_footprint_bound_covers_the_allocation():
    """The admission bound is at least what a shot really holds on the device."""
    import torch
    from ertm_b200.batch import shot_device_bytes
    from ertm_b200.imaging import ShotMigrator
    from ertm_b200.serving import shot_footprint_bound
    for case in CASES:
        job = _job(case, 1)
        mig = ShotMigrator(job.imager, job.model)
        shot = job.shots[0]
        n_comp = len(shot.components)
        nt = int(job.imager.solver_config.nt)
        real = shot_device_bytes(mig, nt, len(job.modes)) + n_comp * nt * shot.data.shape[1] * 4
        assert shot_footprint_bound(job.model, job.imager, nt, len(job.modes), n_comp, shot.data.shape[1]) >= real
    torch.cuda.synchronize()
