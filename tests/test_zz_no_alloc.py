"""The allocation-free LETKF entry point (lbl_letkf_analysis_noalloc) against the
regular one (lbl_assimilate).

Callers that own all their GPU buffers, such as a framework with its own caching
allocator or memory budget, cannot let a library call cudaMalloc.  This entry
point takes their device buffers for the forecast, the observations and the
outputs, and keeps its scratch in a static device array.  Here torch owns the
caller's buffers; the library allocates nothing for the call.  Two calls in a
row, on different ensembles, must reproduce the regular entry point's analysis,
because the shared scratch keeps the previous call's contents.
"""
import ctypes

import numpy as np
import pytest

import lbl

pytestmark = pytest.mark.gpu

P = 4
ANALYSIS_TOL = 1e-5  # relative population tolerance of the analysis parity tests


def make_case(seed, steps):
    cfg = lbl.config_default("DA_LETKF", 64, 8, da_xyprune=P, letkf_rloc_len=1, letkf_covinf=1.1,
                             obs_error_u=0.002, obs_error_rho=1e-4, daprune=1)
    e = lbl.Ensemble(cfg)
    e.init(seed)
    e.update(0, steps)
    nat = lbl.Ensemble(lbl.config_default("NATURE", 64, 1))
    nat.init(0)
    nat.update(0, steps)
    r, u, v, _ = nat.get_fields(0)
    rng = np.random.default_rng(seed)
    obs = [(a + s * rng.standard_normal(a.shape)).astype(np.float32)
           for a, s in ((r, 1e-4), (u, 2e-3), (v, 2e-3))]
    return cfg, e, obs


def sites(a):
    return a[::P, ::P].reshape(-1)


def _call(lib, cfg, d_in, d_out, d_mac, d_yo, stream):
    stats = (ctypes.c_int * 4)()
    err = ctypes.create_string_buffer(256)
    rc = lib.lbl_letkf_analysis_noalloc(ctypes.byref(cfg), ctypes.c_void_p(d_in.data_ptr()),
                                        ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(d_mac.data_ptr()),
                                        ctypes.c_void_p(d_yo.data_ptr()), ctypes.c_void_p(stream.cuda_stream),
                                        stats, err, 256)
    assert rc == 0, (rc, err.value)
    return list(stats)


def test_noalloc_analysis_matches_regular_entry_point():
    torch = pytest.importorskip("torch")
    lib = lbl.load_library()
    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    # the regular entry point's analyses of two different ensembles; the caller's
    # device buffers for both calls are made (by torch) before any call is timed
    cases = []
    for seed, steps in ((0, 20), (3, 35)):
        cfg, e, (ro, uo, vo) = make_case(seed, steps)
        M = cfg.n_ens
        f_in = np.stack([e.get_f(m) for m in range(M)])
        e.assimilate(cfg.iiter, ro, uo, vo)
        want = np.stack([e.get_f(m) for m in range(M)])
        want_u = np.stack([e.get_fields(m)[1] for m in range(M)])
        e.close()
        d_in = torch.from_numpy(f_in).to(dev)
        cases.append(dict(cfg=cfg, want=want, want_u=want_u, d_in=d_in,
                          d_out=torch.full_like(d_in, float("nan")),
                          d_mac=torch.zeros((M, 3, cfg.ny, cfg.nx), dtype=torch.float32, device=dev),
                          d_yo=torch.from_numpy(np.concatenate([sites(uo), sites(vo), sites(ro)])).to(dev)))
    torch.cuda.synchronize()
    # the first call on a device loads the static scratch (set-up); then two calls in a
    # row must leave the device's free memory and torch's allocation where they were
    c0 = cases[0]
    _call(lib, c0["cfg"], c0["d_in"], c0["d_out"], c0["d_mac"], c0["d_yo"], stream)
    torch.cuda.synchronize()
    free0, alloc0 = torch.cuda.mem_get_info(dev)[0], torch.cuda.memory_allocated(dev)
    for call, c in enumerate(cases):
        c["d_out"].fill_(float("nan"))
        stats = _call(lib, c["cfg"], c["d_in"], c["d_out"], c["d_mac"], c["d_yo"], stream)
        torch.cuda.synchronize()
        assert stats[2] == 0 and stats[1] == 0 and stats[0] >= 1, (call, stats)
        got = c["d_out"].cpu().numpy()
        assert np.max(np.abs(got.astype(np.float64) - c["want"]) / np.abs(c["want"])) < ANALYSIS_TOL, call
        mac = c["d_mac"].cpu().numpy()
        np.testing.assert_allclose(mac[:, 1], c["want_u"], rtol=1e-5, atol=1e-7)  # analysis u
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free0, "the allocation-free entry point changed free device memory"
    assert torch.cuda.memory_allocated(dev) == alloc0


def test_noalloc_rejects_oversized_configuration():
    lib = lbl.load_library()
    cfg = lbl.config_default("DA_LETKF", 1024, 32, da_xyprune=1)  # 3*1024^2*32 floats of scratch
    err = ctypes.create_string_buffer(256)
    rc = lib.lbl_letkf_analysis_noalloc(ctypes.byref(cfg), ctypes.c_void_p(1), ctypes.c_void_p(1),
                                        ctypes.c_void_p(1), ctypes.c_void_p(1), None, None, err, 256)
    assert rc == -8
    assert b"scratch" in err.value
