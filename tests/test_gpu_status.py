"""Device-side failure status: a wavefield that becomes NaN or infinite.

The stress phase of every engine sets the propagator's status word when it
writes a non-finite value.  The failures here are made on the host only:
states and shot records whose finite values are near the float32 limit, so
that the propagation overflows within a few steps.  No GPU fault is
involved; the kernels run normally and report through the status word.

* a propagator whose field overflows reports it, a healthy one does not, and
  reset() clears the word;
* the plain and batched migrations raise NonFiniteWavefieldError naming the
  shot;
* in the serving loop the job with the overflowing shot fails alone, while
  the jobs around it return the same images as served alone.
"""

from __future__ import annotations

import numpy as np
import pytest

from test_gpu_serving import _job, _serve

pytestmark = pytest.mark.gpu

HUGE = 3.0e38


def _overflowing(job, shot: int = 0):
    """The job with one shot's record replaced by huge finite values."""
    from dataclasses import replace

    from ertm_b200.serving import ServeJob
    shots = list(job.shots)
    s = shots[shot]
    comps = {k: np.full_like(v, HUGE) for k, v in s.components.items()}
    shots[shot] = replace(s, data=comps[next(iter(comps))], components=comps)
    return ServeJob(shots=shots, model=job.model, imager=job.imager, modes=job.modes, name=job.name + " (overflow)")


@pytest.mark.parametrize("engine", ["acoustic", "elastic", "viscoacoustic"])
def test_propagator_reports_overflow_and_reset_clears_it(engine):
    from ertm_b200.propagation import PropagationSpec, QOptions, build_propagator
    from ertm_b200.types import ElasticModel, GridSpec
    g = GridSpec(nx=60, nz=50, dx=10.0, dz=10.0)
    vp = np.full(g.shape, 2500.0, np.float32)
    model = ElasticModel(grid=g, vp=vp, vs=(vp / 1.8).astype(np.float32), rho=np.full(g.shape, 2100.0, np.float32),
                         qp=np.full(g.shape, 60.0, np.float32), qs=np.full(g.shape, 30.0, np.float32))
    spec = PropagationSpec(dt=1e-3, nt=40, npml=10, boundary="cpml")
    q = QOptions(enabled=True, f_ref=25.0) if engine == "viscoacoustic" else None
    prop = build_propagator(model, spec, engine=engine, q_options=q)
    for _ in range(5):
        prop.step(1.0)
    assert prop.status == 0 and prop.finite
    state = prop.state()
    key = "p" if engine != "elastic" else "sxx"
    zz, xx = np.indices(state[key].shape)
    checker = np.where((zz + xx) % 2 == 0, HUGE, -HUGE).astype(np.float32)   # steep gradients everywhere
    state[key] = checker
    if engine == "viscoacoustic":
        state["eps"] = checker
    prop.load_state(state)
    for _ in range(8):
        prop.step(0.0)
    assert not prop.finite
    prop.reset()
    assert prop.status == 0


def test_plain_migrate_raises_on_overflow():
    from ertm_b200 import NonFiniteWavefieldError
    job = _overflowing(_job("mig_acoustic_zerolag", 1))
    with pytest.raises(NonFiniteWavefieldError):
        job.imager.migrate(job.shots[0], job.model)


def test_batched_migrate_names_the_failed_shot():
    from ertm_b200 import NonFiniteWavefieldError
    from ertm_b200.batch import BatchMigrator
    job = _overflowing(_job("mig_acoustic_zerolag", 3), shot=1)
    with pytest.raises(NonFiniteWavefieldError, match=r"shot\(s\) 1 "):
        BatchMigrator(job.imager).migrate_shots(job.shots, job.model)


def test_serving_fails_the_overflowing_job_alone():
    from ertm_b200 import NonFiniteWavefieldError
    from ertm_b200.serving import RTMServer
    good = [_job("mig_acoustic_zerolag"), _job("mig_elastic_pp_divcurl"), _job("mig_visco_comp")]
    bad = _overflowing(_job("mig_acoustic_norm_rn"), shot=1)
    alone = [_serve([j])[0][0] for j in good]
    with RTMServer(max_shots=4, ticks_per_poll=5) as srv:
        futs = [srv.submit(j) for j in (good[0], bad, good[1], good[2])]
        with pytest.raises(NonFiniteWavefieldError):
            futs[1].result(timeout=600)
        served = [futs[k].result(timeout=600) for k in (0, 2, 3)]
    for a, m in zip(alone, served):
        for x, y in zip(a.images, m.images):
            assert np.array_equal(x.image, y.image), a.name
    s = srv.summary()
    assert s["jobs_failed"] == 1 and s["jobs_done"] == 3 and s.get("shots_failed", 0) >= 1
