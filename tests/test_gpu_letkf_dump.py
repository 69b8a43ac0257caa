"""LETKF matrix dumps (need_save_mat, letkf.cu:33 and letkf_solver.h:243-345): file
names and shapes per reference rank, HDF5 structure, and the algebra that ties the
14 matrices together and to the analysis the engine applied."""
import os

import numpy as np
import pytest

import lbl
import oracle
from h5_parse import read_datasets
from test_gpu_letkf import make_case

pytestmark = pytest.mark.gpu

LABELS = ["_dYf", "_dyo", "_Q", "_V", "_Xf", "_dXf", "_Pa", "_dWa", "_Xa", "_Wa", "_AI", "_Z", "_Lambda", "_Wma"]


def load(d, label, t):
    names = [n for n in os.listdir(d) if n.startswith(label + ".float_") and n.endswith(f".{t}.h5")]
    assert len(names) == 1, (label, names)
    a = read_datasets(os.path.join(d, names[0]))["data"]
    rows, cols, nb = (int(x) for x in names[0][len(label) + 7:].split(".")[0].split("_"))
    assert a.shape == (rows, cols, nb)
    # the buffer is column-major per matrix with the point slowest (cu_matrix.hpp:53)
    return np.asarray(a).reshape(-1).reshape(nb, cols, rows).transpose(0, 2, 1).astype(np.float64)


def test_matrix_dumps(tmp_path):
    nx, M, p, L, beta = 64, 8, 4, 1, 1.1
    cfg, e, obs, _, _ = make_case(nx, M, p, L, beta, write_mat=1)
    e.set_io_prefix(str(tmp_path))
    F = np.stack([e.get_f(m) for m in range(M)]).astype(np.float64)      # [M][9][ny][nx]
    t = cfg.iiter
    e.assimilate(t, *obs)
    Fa = np.stack([e.get_f(m) for m in range(M)]).astype(np.float64)
    o = oracle.Oracle(cfg)
    nobs = 3 * (2 * 2 * L + 1) ** 2
    rows = nx // M
    nb = rows * nx
    for r in range(M):
        d = tmp_path / "letkf" / "mat" / f"ens{r}"
        assert sorted(n.split(".")[0] for n in os.listdir(d)) == sorted(LABELS)
        m = {lab: load(str(d), lab, t) for lab in LABELS}
        assert m["_dYf"].shape == (nb, nobs, M) and m["_dyo"].shape == (nb, nobs, 1)
        pts = np.arange(r * nb, (r + 1) * nb)
        Xf = F.reshape(M, 9, -1)[:, :, pts].transpose(2, 1, 0)              # [b][q][k]
        Xa = Fa.reshape(M, 9, -1)[:, :, pts].transpose(2, 1, 0)
        np.testing.assert_array_equal(m["_Xf"], Xf)                       # the forecast
        np.testing.assert_array_equal(m["_Xa"], Xa)                       # the analysis the engine wrote
        np.testing.assert_allclose(m["_AI"], Xa - Xf, rtol=0, atol=1e-7)
        np.testing.assert_allclose(m["_dXf"], Xf - Xf.mean(2, keepdims=True), rtol=0, atol=1e-6)
        Q, V, Lam = m["_Q"], m["_V"], m["_Lambda"]
        scale = np.abs(Q).max()
        np.testing.assert_allclose(Q, Q.transpose(0, 2, 1), rtol=0, atol=1e-5 * scale)
        eye = np.eye(M)
        np.testing.assert_allclose(V.transpose(0, 2, 1) @ V, np.broadcast_to(eye, V.shape), atol=1e-5)
        np.testing.assert_allclose(Q @ V, V @ Lam, rtol=0, atol=1e-4 * scale)
        np.testing.assert_allclose(m["_Pa"] @ Q, np.broadcast_to(eye, Q.shape), atol=1e-4)
        dW = m["_dWa"]
        np.testing.assert_allclose(dW @ dW @ Q / (M - 1), np.broadcast_to(eye, Q.shape), atol=1e-4)
        np.testing.assert_allclose(m["_Wa"], dW + m["_Wma"], rtol=0, atol=1e-6)
        np.testing.assert_allclose(m["_Z"], m["_Wa"] - eye, rtol=0, atol=1e-6)
        assert np.all(m["_Wma"] == m["_Wma"][:, :, :1])                   # w 1^T: equal columns
        np.testing.assert_allclose(Xa, Xf.mean(2, keepdims=True) + m["_dXf"] @ m["_Wa"], rtol=0, atol=1e-6)
        # the Gram from the dumped window and the reference's R^-1 x Gaspari-Cohn weights
        for b in (0, nb // 3, nb - 1):
            i, j = (r * nb + b) % nx, (r * nb + b) // nx
            w = np.zeros(nobs)
            nox = int(round(np.sqrt(nobs // 3)))
            for var in range(3):
                for bb in range(nox):
                    for aa in range(nox):
                        wt, valid = o.obs_weight(i, j, aa, bb, var)
                        w[aa + nox * bb + var * nox * nox] = wt if valid else 0.0
            dY = m["_dYf"][b]
            Qe = (M - 1) / beta * eye + dY.T @ (w[:, None] * dY)
            np.testing.assert_allclose(Q[b], Qe, rtol=0, atol=1e-5 * np.abs(Qe).max())
    o.close()


def test_write_mat_needs_whole_rows_per_rank():
    with pytest.raises(lbl.LblError) as ei:
        lbl.Ensemble(lbl.config_default("DA_LETKF", 64, 6, da_xyprune=4, write_mat=1))
    assert ei.value.code == -1
