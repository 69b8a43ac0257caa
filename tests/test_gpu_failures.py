"""Failure paths through the C ABI, made on the host or by a bounded wait that runs
out -- none faults, traps or hangs the GPU:

* missing and short observation files for lbl_assimilate_files (the read path of
  src/letkf.cu:197-220, which throws on them) -> LBL_ERR_IO, context still usable;
* a context larger than the device -> LBL_ERR_NOMEM with every partial allocation
  returned (free device memory unchanged afterwards);
* the TMA stream-collide with its producer told to issue nothing and a short poll
  limit (lbl_inject): the consumers' bounded waits give up, nothing is in flight, the
  call returns LBL_ERR_TIMEOUT, and after lbl_init the context steps again.
"""
import os

import numpy as np
import pytest

import lbl

pytestmark = pytest.mark.gpu

ERR_IO, ERR_NOMEM, ERR_TIMEOUT = -4, -7, -10


def _write(path, a):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.ascontiguousarray(a, np.float32).tofile(path)


def test_missing_and_short_observation_files(tmp_path):
    cfg = lbl.config_default("DA_LETKF", 64, 4, da_xyprune=4, letkf_rloc_len=1, letkf_covinf=1.1, daprune=1)
    e = lbl.Ensemble(cfg)
    e.init(0)
    e.update(0, cfg.iiter)
    t = cfg.iiter
    step = t // cfg.iiter
    obs_dir = tmp_path / "io" / "observed" / "ens0000"
    name = lambda v: str(obs_dir / f"{v}_step{step:010d}.dat")  # noqa: E731
    f0 = [e.get_f(m) for m in range(cfg.n_ens)]
    # no files at all
    with pytest.raises(lbl.LblError) as ei:
        e.assimilate_files(t, str(tmp_path / "io"))
    assert ei.value.code == ERR_IO and "could not open" in str(ei.value)
    # rho present, u short by one value, v missing
    r, u, v, _ = e.get_fields(0)
    _write(name("rho"), r)
    _write(name("u"), u.reshape(-1)[:-1])
    with pytest.raises(lbl.LblError) as ei:
        e.assimilate_files(t, str(tmp_path / "io"))
    assert ei.value.code == ERR_IO and "short read" in str(ei.value)
    # the failed calls left the ensemble as it was
    for m in range(cfg.n_ens):
        np.testing.assert_array_equal(e.get_f(m), f0[m])
    # complete files: the analysis runs
    _write(name("u"), u)
    _write(name("v"), v)
    e.assimilate_files(t, str(tmp_path / "io"))
    assert e.letkf_stats()["max_sweeps"] >= 1
    assert any(np.any(e.get_f(m) != f0[m]) for m in range(cfg.n_ens))
    e.close()


def test_allocation_failure_returns_nomem_without_leak():
    torch = pytest.importorskip("torch")
    warm = lbl.Ensemble(lbl.config_default("NATURE", 64, 2))  # loads the library's device code first
    warm.close()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    # NATURE at 1024^2 with 2700 members: each population buffer is 102 GB and each macro
    # buffer 34 GB, so the first buffers fit in the device and the second population
    # buffer does not
    cfg = lbl.config_default("NATURE", 1024, 2700)
    with pytest.raises(lbl.LblError) as ei:
        lbl.Ensemble(cfg)
    assert ei.value.code == ERR_NOMEM, ei.value
    torch.cuda.synchronize()
    # (a context released just before may return a few MiB late, so free memory may grow)
    assert torch.cuda.mem_get_info(0)[0] >= free0, "allocations of the failed context were not returned"
    # the failure is not sticky: a normal context works afterwards
    e = lbl.Ensemble(lbl.config_default("NATURE", 64, 2))
    e.init(0)
    e.update(0, 3)
    e.close()


def test_tma_wait_timeout_is_reported():
    """A direct-load context takes the same calls, so both draw the same forcing normals
    (lbl_init resets the cursor, not the cuRAND generator)."""
    ctxs = [lbl.Ensemble(lbl.config_default("NATURE", 64, 2, lbm_variant=v)) for v in (lbl.LBM_TMA, lbl.LBM_DIRECT)]
    for e in ctxs:
        e.init(0)
        e.update(0, 2)
    tma, ref = ctxs
    tma.inject(lbl.INJECT_TMA_STALL, 256)
    with pytest.raises(lbl.LblError) as ei:
        tma.update(0, 1)
    assert ei.value.code == ERR_TIMEOUT and "gave up" in str(ei.value)
    ref.update(0, 1)
    tma.inject(lbl.INJECT_NONE)
    for e in ctxs:
        e.init(0)
        e.update(0, 5)
    for m in range(2):
        np.testing.assert_allclose(tma.get_f(m), ref.get_f(m), rtol=1e-6, atol=1e-7)
    for e in ctxs:
        e.close()
