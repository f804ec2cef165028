"""WPM with the bins split across CTA groups (few probes) against the fused
kernels (many probes): the blend of a pixel adds the same two weighted fields
in the same order and the transforms are the same code, so a probe gives the
same wave alone (split) and inside a large batch (fused)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wap():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import wideanglepropagation_b200 as w
    return w


@pytest.mark.parametrize("K", [16, 7])
def test_split_bins_match_fused(wap, K):
    import wideanglepropagation_b200.synthetic as S
    w = S.batched_scan_class(2, 128, 4, 8, 1)             # 64 probes on 128^2
    dev = torch.device("cuda")
    V = torch.as_tensor(w.potential, device=dev)
    probe = torch.as_tensor(w.probe, device=dev)
    pos = torch.as_tensor(w.positions, device=dev)
    kw = dict(n_bins=K, power_spacing=1.5)
    ex_all, dp_all, st_all = wap.simulate_wpm(V[0], probe, w.dz, w.energy, (w.ps, w.ps), positions=pos, **kw)
    for b in (0, 37):
        ex, dp, st = wap.simulate_wpm(V[0], probe, w.dz, w.energy, (w.ps, w.ps), positions=pos[b:b + 1], **kw)
        assert float((ex[0] - ex_all[b]).norm() / ex_all[b].norm()) < 1e-6
        assert float((dp[0] - dp_all[b]).norm() / dp_all[b].norm()) < 1e-6
        assert float((st[0] - st_all[b]).norm() / st_all[b].norm()) < 1e-6   # every slice's snapshot


def test_split_bins_match_oracle(wap):
    """A single 256^2 probe (split path) against the FP64 oracle."""
    import wideanglepropagation_b200.synthetic as S
    from oracle import propagation_oracle as O
    w = S.wpm_fcc(1, n_slices=6, n=256)
    ex, dp, _ = wap.simulate_wpm(w.potential[0], w.probe, w.dz, w.energy, (w.ps, w.ps), 16, 1.0)
    ref = O.simulate_wpm(w.potential[0].astype(np.float64), w.probe, w.dz, w.energy, (w.ps, w.ps), 16, 1.0,
                         return_wavefronts=False)
    assert O.rel_l2(ex.cpu().numpy(), ref[0]) < 1e-5
    assert O.rel_l2(dp.cpu().numpy(), ref[1]) < 1e-5
