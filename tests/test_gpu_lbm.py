"""Forecast path on the GPU, through the C ABI, against the reference's own run
(golden fixtures) and the FP64 oracle: initial condition, forcing (cuRAND stream,
cursor, field), fused stream-collide, macros, graphs and chunking."""
import os

import numpy as np
import pytest

from conftest import checksums, golden, rel_err

import lbl
import oracle

pytestmark = pytest.mark.gpu
N4 = 4 * 29


def nature(nx=256, M=1, ofs=0, **kw):
    e = lbl.Ensemble(lbl.config_default("NATURE", nx, M, **kw))
    e.init(ofs)
    return e


def test_initial_condition_matches_oracle_bitwise():
    e = nature(256)
    r, u, v, f = oracle.ic_fields(e.cfg, 0)
    np.testing.assert_array_max_ulp(e.get_f(0), f, maxulp=2)
    rr, uu, vv, _ = e.get_fields(0)
    np.testing.assert_array_max_ulp(uu, u, maxulp=2)
    np.testing.assert_array_max_ulp(vv, v, maxulp=2)
    np.testing.assert_array_equal(rr, r)


@pytest.mark.parametrize("name,mode,seed_member", [("ref_lbm_id0.npz", "NATURE", 0), ("ref_lbm_id334.npz", "DA_LETKF", 0)])
def test_initial_condition_matches_reference(name, mode, seed_member):
    g = golden(name)
    e = lbl.Ensemble(lbl.config_default(mode, 256, 2))
    e.init(0)
    f = e.get_f(seed_member)
    rows = g["rows"]
    np.testing.assert_array_max_ulp(f[:, rows, :], g["s0_rows_f"], maxulp=1)
    np.testing.assert_allclose(checksums(f), g["s0_sums_f"], rtol=1e-7)


def test_forcing_stream_and_cursor_match_reference():
    g = golden("ref_lbm_id0.npz")
    e = nature(256)
    st = e.force_state()
    np.testing.assert_array_equal(st["kx"], g["kx"])
    np.testing.assert_array_equal(st["amp"], g["amp"])
    assert st["cursor"] == int(g["s0_cursor"][0]) == N4
    np.testing.assert_array_equal(st["randoms"], g["normals_head"][N4:2 * N4])  # cuRAND MTGP32, seed 1991
    e.update(0, 1)
    st = e.force_state()
    assert st["cursor"] == int(g["s1_cursor"][0])
    np.testing.assert_array_equal(st["randoms"], g["normals_head"][2 * N4:3 * N4])
    fx, fy = e.force()
    rows = g["rows"]
    np.testing.assert_array_equal(fx[rows], g["s1_rows_fx"])  # bit-exact
    np.testing.assert_array_equal(fy[rows], g["s1_rows_fy"])


def test_steps_match_reference_within_1e5():
    """Populations after 1, 10 and 100 steps within 1e-5 relative of the reference's.

    "Relative" is the normwise error ||f - f_ref|| / ||f_ref|| over the fixture rows.  The
    elementwise max |df|/|f| is also bounded, at 3e-5: the reference's FP32 rounding is
    not reproducible at the bit level even by the reference itself (its own lbm.h moment
    functions compiled outside its fused streaming kernel round differently), and with
    omega ~ 2 rounding noise is not damped, so the reference sits 1.2e-5 elementwise from
    the FP64 oracle after 100 steps (tests/test_oracle_golden.py)."""
    g = golden("ref_lbm_id0.npz")
    e = nature(256)
    rows = g["rows"]
    done = 0
    worst = {}
    for s in sorted(int(x) for x in g["steps"]):
        if s > done:
            e.update(done, s - done)
            done = s
        f = e.get_f(0).astype(np.float64)
        ref = g[f"s{s}_rows_f"].astype(np.float64)
        d = f[:, rows, :] - ref
        norm = float(np.linalg.norm(d) / np.linalg.norm(ref))
        elem = float(np.max(np.abs(d) / np.abs(ref)))
        worst[s] = (norm, elem)
        assert norm < 1e-5, (s, norm)
        assert elem < 3e-5, (s, elem)
        np.testing.assert_allclose(checksums(f), g[f"s{s}_sums_f"], rtol=1e-6)
        if s > 0:
            # the forcing of step s is bit-exact (the chunks here are 1, 9 and 90 steps)
            fx, fy = e.force()
            np.testing.assert_array_equal(fx[rows], g[f"s{s}_rows_fx"])
            np.testing.assert_array_equal(fy[rows], g[f"s{s}_rows_fy"])
            # u = c*sum(f e_x)/rho cancels O(0.1) populations down to O(1e-3): a 1e-5 bound on
            # f allows ~1e-3 of max|u|; rho = sum(f) keeps the population bound
            r, u, v, _ = e.get_fields(0)
            assert rel_err(u[rows], g[f"s{s}_rows_u"]) < 1e-3
            assert rel_err(v[rows], g[f"s{s}_rows_v"]) < 1e-3
            assert rel_err(r[rows], g[f"s{s}_rows_r"]) < 1e-5
    print("population error vs reference per step (normwise, elementwise max):", worst)


@pytest.mark.parametrize("kf", [4.0, 8.0])  # 29 modes (register kernel), 61 (per-step kernel)
def test_forcing_field_matches_oracle(kf):
    e = nature(128, M=1, kf=kf)
    o = oracle.Oracle(e.cfg)
    assert (e.force_state()["n_modes"] <= 32) == (kf == 4.0)
    for _ in range(3):
        e.update(0, 1)
        st = e.force_state()
        fx, fy = e.force()
        ofx, ofy = o.force(st["randoms"])
        assert rel_err(fx, ofx) < 2e-5
        assert rel_err(fy, ofy) < 2e-5


def test_stream_collide_matches_fp64_oracle():
    """Engine forces injected into the oracle each step; 50 steps, 3 members."""
    e = nature(128, M=3, ofs=5)
    o = oracle.Oracle(e.cfg)
    for m in range(3):
        o.set_f(m, e.get_f(m))
    for t in range(50):
        e.update(t, 1)
        fx, fy = e.force()
        o.set_force(fx, fy)
        o.step_noforce()
    for m in range(3):
        fe, fo = e.get_f(m).astype(np.float64), o.get_f(m)
        assert np.max(np.abs(fe - fo) / np.abs(fo)) < 1e-5
        r, u, v, _ = e.get_fields(m)
        ro, uo, vo = o.macros(m)
        assert rel_err(u, uo) < 1e-3 and rel_err(v, vo) < 1e-3
        assert rel_err(r, ro) < 1e-5  # FP32 storage of f vs FP64 over 50 steps


def test_chunking_and_graphs_are_bitwise_invariant():
    a = nature(128, M=2)
    b = nature(128, M=2)
    a.update(0, 37)
    for t in range(37):
        b.update(t, 1)
    for m in range(2):
        np.testing.assert_array_equal(a.get_f(m), b.get_f(m))
        np.testing.assert_array_equal(a.get_fields(m)[2], b.get_fields(m)[2])


def test_members_are_independent_runs():
    big = nature(128, M=3)
    big.update(0, 10)
    for k in range(3):
        one = nature(128, M=1, ofs=k)
        one.update(0, 10)
        np.testing.assert_array_equal(big.get_f(k), one.get_f(0))


def test_long_run_crosses_normal_refill():
    """1100 steps cross the 1023-call refill of the cuRAND buffer (data.cu:241-247)."""
    e = nature(64, M=1)
    e.update(0, 1100)
    st = e.force_state()
    assert st["cursor"] == ((2 + 1100 - 1) % 1023) * N4
    f = e.get_f(0)
    assert np.all(np.isfinite(f))


def test_diagnostics_fp64():
    e = nature(128, M=2)
    e.update(0, 5)
    r, u, v, w = e.get_fields(1)
    d = e.diagnostics(1)
    np.testing.assert_allclose(d["energy"], 0.5 * np.mean(u.astype(np.float64) ** 2 + v.astype(np.float64) ** 2), rtol=1e-9)
    np.testing.assert_allclose(d["mass"], np.mean(r.astype(np.float64)), rtol=1e-12)
    np.testing.assert_allclose(d["enstrophy"], 0.5 * np.mean(w.astype(np.float64) ** 2), rtol=1e-4)


def test_errors_are_reported_not_crashed():
    with pytest.raises(lbl.LblError) as ei:
        lbl.Ensemble(lbl.config_default("NATURE", 100, 1))
    assert ei.value.code == -1
    with pytest.raises(lbl.LblError) as ei:
        lbl.Ensemble(lbl.config_default("DA_LETKF", 64, 1))
    assert ei.value.code == -8
    e = lbl.Ensemble(lbl.config_default("NATURE", 64, 1))
    with pytest.raises(lbl.LblError) as ei:
        e.update(0, 1)
    assert ei.value.code == -6


@pytest.mark.parametrize("nx", [64, 256, 512])
def test_stream_collide_variants_agree(nx):
    """The TMA-fed and the direct-load stream-collide compute the same arithmetic."""
    out = {}
    for variant in (lbl.LBM_DIRECT, lbl.LBM_TMA):
        e = lbl.Ensemble(lbl.config_default("NATURE", nx, 2, lbm_variant=variant))
        e.init(0)
        e.update(0, 25)
        out[variant] = [e.get_f(m).astype(np.float64) for m in range(2)] + [e.get_fields(1)[1]]
    # the two kernels are the same arithmetic, contracted into FMAs independently by the
    # compiler; with omega ~ 2 last-bit differences are not damped over the 25 steps
    for a, b in zip(out[lbl.LBM_DIRECT][:2], out[lbl.LBM_TMA][:2]):
        assert np.linalg.norm(a - b) / np.linalg.norm(a) < 1e-6
        assert np.max(np.abs(a - b) / np.abs(a)) < 1e-5
    # u = c*sum(f e_x)/rho cancels O(0.1) populations, so it is bounded against max|u|
    ud = out[lbl.LBM_DIRECT][2]
    np.testing.assert_allclose(out[lbl.LBM_TMA][2], ud, rtol=0, atol=1e-4 * np.max(np.abs(ud)))


@pytest.mark.parametrize("nx,ny,members,variant,storage", [
    (64, 64, 3, "LBM_VEC", 0), (64, 64, 3, "LBM_VEC2", 0), (128, 128, 2, "LBM_VEC", 0), (256, 256, 2, "LBM_VEC", 0),
    (256, 256, 2, "LBM_VEC2", 0), (96, 40, 2, "LBM_VEC", 0), (32, 8, 2, "LBM_VEC", 0), (512, 512, 1, "LBM_VEC", 0),
    (1024, 64, 1, "LBM_VEC2", 0), (256, 256, 2, "LBM_VEC2", 1), (512, 512, 1, "LBM_VEC", 1), (96, 40, 2, "LBM_VEC2", 1),
    (64, 64, 3, "LBM_VEC", 1)])
def test_vector_stream_collide_is_bit_identical(nx, ny, members, variant, storage):
    """The vector-load stream-collide (4 or 2 columns per thread) does each cell's
    arithmetic in the same explicitly rounded sequence as the one-column kernel, so
    populations and macros agree bit for bit, in FP32 and in FP16 deviation storage,
    with and without the prefetched row and whatever the strip height.  The sizes
    cover every compiled grid width and the run-time one (96 x 40, 1024 x 64, and
    32 x 8, where one thread holds a quarter of the row)."""
    out = {}
    cfg = dict(ny=ny, storage=storage)
    e = lbl.Ensemble(lbl.config_default("NATURE", nx, members, lbm_variant=lbl.LBM_DIRECT, **cfg))
    e.init(0)
    e.update(0, 25)
    ref = [e.get_f(m) for m in range(members)] + [a for m in range(members) for a in e.get_fields(m)[:3]]
    e.close()
    for prefetch, strip in ((True, 0), (False, 0), (True, 5), (False, 3)):
        e = lbl.Ensemble(lbl.config_default("NATURE", nx, members, lbm_variant=getattr(lbl, variant), **cfg))
        e.set_launch_shape(prefetch, strip)
        shape = e.launch_shape()
        assert shape["columns_per_thread"] == (4 if variant == "LBM_VEC" else 2) and shape["prefetch"] == prefetch
        e.init(0)
        e.update(0, 25)
        out = [e.get_f(m) for m in range(members)] + [a for m in range(members) for a in e.get_fields(m)[:3]]
        e.close()
        for a, b in zip(ref, out):
            np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("nx,members,storage", [(128, 4, 0), (256, 2, 1)])
def test_autotuned_shape_is_reported_and_bit_identical(nx, members, storage):
    """lbl_autotune on an LBL_LBM_AUTO context picks the columns per thread (1, 2 or 4),
    the march form and the strip height; lbl_stream_collide_shape reports the pick, and
    the run equals the one-column kernel's bit for bit."""
    ref = lbl.Ensemble(lbl.config_default("NATURE", nx, members, lbm_variant=lbl.LBM_DIRECT, storage=storage))
    ref.init(0)
    ref.update(0, 30)
    e = lbl.Ensemble(lbl.config_default("NATURE", nx, members, storage=storage))
    ty, ms = e.autotune()
    shape = e.launch_shape()
    assert shape["columns_per_thread"] in (1, 2, 4) and shape["strip_rows"] == ty and ms > 0
    assert shape["prefetch"] or shape["columns_per_thread"] > 1
    e.init(0)
    e.update(0, 30)
    for m in range(members):
        np.testing.assert_array_equal(e.get_f(m), ref.get_f(m))
    e.close()
    ref.close()


def test_vector_stream_collide_rejects_what_it_does_not_serve():
    with pytest.raises(lbl.LblError, match="nx <= 1024"):
        lbl.Ensemble(lbl.config_default("NATURE", 2048, 1, lbm_variant=lbl.LBM_VEC))
    e = lbl.Ensemble(lbl.config_default("NATURE", 64, 1, lbm_variant=lbl.LBM_DIRECT))
    with pytest.raises(lbl.LblError, match="without prefetch"):
        e.set_launch_shape(False, 0)
    with pytest.raises(lbl.LblError, match="strip_rows"):
        e.set_launch_shape(True, 65)
    e.close()


@pytest.mark.parametrize("fixture,physics", [("ref_longrun_id0.npz", {}),
                                             ("ref_longrun_c0_id0.npz", dict(cs=0.1, tau=0.51))])
def test_long_run_statistics_match_reference(fixture, physics):
    """10,000 steps of the NATURE case against the reference's own build run for the
    same 10,000 steps (tests/golden/make_longrun.py): kinetic energy, enstrophy and
    the energy spectrum in octave bands, sampled every 500 steps from step 2000.  A
    chaotic run may only be compared in such statistics; the bound is 2e-3 relative
    (the requirement is 2 %), and the measured agreement is about 1e-4.  Two physics:
    the reference's defaults (Cs 0.2, nu 1e-4), and the C0 nature run's Cs 0.1 and
    tau 0.51 (the reference built from a patched copy, oracle/make_ref_c0.sh), both
    from the reference's band-limited initial condition."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    import make_longrun as ml
    g = golden(fixture)
    dx = float(np.float32(2 * np.pi) / np.float32(255))
    e = nature(256, **physics)
    spectra, energy, enstrophy, t = [], [], [], 0
    for s in g["steps"]:
        e.update(t, int(s) - t)
        t = int(s)
        _, u, v, _ = e.get_fields(0)
        sp, en, z = ml.stats(u, v, dx)
        spectra.append(sp)
        energy.append(en)
        enstrophy.append(z)
    assert abs(np.mean(energy) / np.mean(g["energy"]) - 1) < 2e-3
    assert abs(np.mean(enstrophy) / np.mean(g["enstrophy"]) - 1) < 2e-3
    mine, ref = np.mean(spectra, 0), g["spectra"].mean(0)
    for k0, k1 in ((1, 4), (4, 8), (8, 16), (16, 32), (32, 64), (64, 128)):
        assert abs(mine[k0:k1].sum() / ref[k0:k1].sum() - 1) < 2e-3, (k0, k1)


@pytest.mark.parametrize("nx,ny,M,steps", [(2048, 16, 2, 20), (1280, 24, 1, 20), (1536, 16, 1, 10), (8192, 8, 1, 10),
                                           (2048, 2048, 1, 2)])
def test_wide_rows_match_fp64_oracle(nx, ny, M, steps):
    """Rows wider than 1024 columns: a cluster of CTAs per strip (2048 = 2 x 1024,
    1280 = 5 x 256, 1536 = 3 x 512, 8192 = 8 x 1024: the widest), the (u, v) across a
    chunk edge read from the neighbour CTA's shared memory."""
    e = lbl.Ensemble(lbl.config_default("NATURE", nx, M, ny=ny))
    e.init(0)
    o = oracle.Oracle(e.cfg)
    for m in range(M):
        o.set_f(m, e.get_f(m))
    for t in range(steps):
        e.update(t, 1)
        fx, fy = e.force()
        o.set_force(fx, fy)
        o.step_noforce()
    for m in range(M):
        fe, fo = e.get_f(m).astype(np.float64), o.get_f(m)
        assert np.max(np.abs(fe - fo) / np.abs(fo)) < 1e-5


def test_wide_rows_limits():
    with pytest.raises(lbl.LblError) as ei:  # a multiple of 32 that no cluster of <= 8 CTAs splits
        lbl.Ensemble(lbl.config_default("NATURE", 2080, 1, ny=16))
    assert ei.value.code == -1
    with pytest.raises(lbl.LblError) as ei:  # the analysis stays at <= 1024 columns
        lbl.Ensemble(lbl.config_default("DA_LETKF", 2048, 2, ny=16))
    assert ei.value.code == -8


def test_tma_variant_rejected_where_unsupported():
    with pytest.raises(lbl.LblError) as ei:
        lbl.Ensemble(lbl.config_default("NATURE", 384, 1, lbm_variant=lbl.LBM_TMA))
    assert ei.value.code == -8



def test_autotune_changes_speed_not_results():
    cfg = lbl.config_default("NATURE", 256, 3)
    a, b = lbl.Ensemble(cfg), lbl.Ensemble(cfg)
    ty, ms = a.autotune()
    assert 2 <= ty <= 64 and ms > 0
    for x in (a, b):
        x.init(0)
        x.update(0, 12)
    for m in range(3):
        np.testing.assert_array_equal(a.get_f(m), b.get_f(m))  # strip height never changes the arithmetic
    with pytest.raises(lbl.LblError) as ei:
        a.autotune()  # only before init
    assert ei.value.code == -6
