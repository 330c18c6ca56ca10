"""CUDA-graph replay and the autotuner (GPU)."""

import numpy as np
import pytest
import torch

import ptyrodactyl_b200 as pb
from oracle import multislice_ref as R
from ptyrodactyl_b200 import synth
from ptyrodactyl_b200.autotune import tune_forward
from ptyrodactyl_b200.graphs import GraphedForward

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    w = synth.CONFIG1
    dev = torch.device("cuda")
    pot = torch.as_tensor(synth.potential_slices(w, num_slices=6), device=dev)
    probe = R.make_probe(w.voltage_kv, w.aperture_mrad, (w.n, w.n), w.calib * 100.0)
    modes = torch.as_tensor(probe[..., None].astype(np.complex64), device=dev)
    wts = torch.ones(1, device=dev)
    pos = torch.as_tensor(synth.raster_positions(w)[:40], device=dev).contiguous()
    return w, pot, modes, wts, pos


def test_graph_replay_matches_direct_and_follows_inputs(case):
    w, pot, modes, wts, pos = case
    g = GraphedForward(pot, modes, wts, pos.clone(), synth.SLICE_DZ, w.voltage_kv, w.calib, batch=16)
    assert g.launches_per_replay > 0
    direct = pb.run_forward(pot, synth.SLICE_DZ, modes, wts, pos, w.voltage_kv, w.calib, w.calib, batch=16)
    out = g.replay().clone()
    torch.cuda.synchronize()
    assert torch.equal(out, direct)
    moved = (pos + 0.75).contiguous()
    g.positions.copy_(moved)
    out2 = g.replay().clone()
    direct2 = pb.run_forward(pot, synth.SLICE_DZ, modes, wts, moved, w.voltage_kv, w.calib, w.calib, batch=16)
    torch.cuda.synchronize()
    assert torch.equal(out2, direct2)
    assert not torch.equal(out2, out)


def test_autotune_picks_and_caches(case, tmp_path, monkeypatch):
    monkeypatch.setenv("PTYRO_B200_TUNE_CACHE", str(tmp_path / "tune.json"))
    import ptyrodactyl_b200.autotune as at
    at._memo.clear()
    w, pot, modes, wts, pos = case
    batch, tune = tune_forward(pot, modes, wts, pos, synth.SLICE_DZ, w.voltage_kv, w.calib)
    from ptyrodactyl_b200.autotune import candidates
    assert (batch, tune) in candidates(pot.shape[0], pos.shape[0], modes.shape[2])
    assert (tmp_path / "tune.json").exists()
    at._memo.clear()
    assert tune_forward(pot, modes, wts, pos, synth.SLICE_DZ, w.voltage_kv, w.calib) == (batch, tune)
    ref = pb.run_forward(pot, synth.SLICE_DZ, modes, wts, pos, w.voltage_kv, w.calib, w.calib)
    got = pb.run_forward(pot, synth.SLICE_DZ, modes, wts, pos, w.voltage_kv, w.calib, w.calib, batch=batch,
                         tune=tune)
    assert torch.equal(ref, got)


def test_lanes_do_not_change_results():
    import numpy as np
    from oracle import multislice_ref as R
    from ptyrodactyl_b200.graphs import GraphedForward
    from ptyrodactyl_b200.simulations import run_forward
    rng = np.random.default_rng(21)
    n, s, p = 64, 5, 37
    dev = torch.device("cuda")
    slices = torch.as_tensor(rng.uniform(0, 40, (n, n, s)), dtype=torch.float32, device=dev)
    probe = R.make_probe(200.0, 25.0, (n, n), 30.0, defocus_ang=-20.0)
    modes = torch.as_tensor(probe[..., None].astype(np.complex64), device=dev)
    wt = torch.ones(1, device=dev)
    pos = torch.as_tensor(rng.uniform(-2, 2, (p, 2)), dtype=torch.float64, device=dev)
    one = run_forward(slices, 1.7, modes, wt, pos, 200.0, 0.3, 0.3, batch=4, lanes=1)
    three = run_forward(slices, 1.7, modes, wt, pos, 200.0, 0.3, 0.3, batch=4, lanes=3)
    assert torch.equal(one, three)
    g = GraphedForward(slices, modes, wt, pos, 1.7, 200.0, 0.3, batch=4, lanes=2)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(g.out, one)


@pytest.mark.parametrize("n", [16, 32, 64, 128, 256, 512])
def test_paired_steady_kernels_are_bit_identical(n):
    """Two-lines-per-thread f32x2 steady passes (tune bits 16, 32, 64, 128; at 256^2
    also 2048: column blocks moved by TMA, 4096: the first and last slice passes
    paired, 16384: line-pair interleaved transmission tables, used where the window
    keeps a pair aligned) give exactly the one-line kernel's patterns, also with
    windows, and no TMA wait gives up."""
    import numpy as np
    from oracle import multislice_ref as R
    from ptyrodactyl_b200.simulations import run_forward
    rng = np.random.default_rng(n)
    s, p = 5, 6
    dev = torch.device("cuda")
    slices = torch.as_tensor(rng.uniform(0, 40, (n, n, s)), dtype=torch.float32, device=dev)
    probe = R.make_probe(200.0, 25.0, (n, n), 30.0, defocus_ang=-20.0)
    modes = torch.as_tensor(np.stack([probe, np.roll(probe, 1, 0)], -1).astype(np.complex64), device=dev)
    wt = torch.tensor([0.6, 0.4], device=dev)
    pos = torch.as_tensor(rng.uniform(-2, 2, (p, 2)), dtype=torch.float64, device=dev)
    ref = run_forward(slices, 1.7, modes, wt, pos, 200.0, 0.3, 0.3, tune=3, lanes=1)
    for tune in (19, 51, 83, 147, 211, 2259, 6355, 4307, 22739):
        got = run_forward(slices, 1.7, modes, wt, pos, 200.0, 0.3, 0.3, tune=tune, lanes=1)
        assert torch.equal(got, ref), tune
    if n <= 256:
        field = torch.as_tensor(rng.uniform(0, 40, (2 * n, 2 * n, s)), dtype=torch.float32, device=dev)
        win = torch.as_tensor(rng.integers(0, 2 * n, (p, 2)), dtype=torch.int32, device=dev)
        ref = run_forward(field, 1.7, modes, wt, pos, 200.0, 0.3, 0.3, tune=3, windows=win, lanes=1)
        for tune in (19, 51, 211, 2259, 6355, 22739):
            got = run_forward(field, 1.7, modes, wt, pos, 200.0, 0.3, 0.3, tune=tune, windows=win, lanes=1)
            assert torch.equal(got, ref), tune
    torch.cuda.synchronize()
    assert pb._lib.load().ptyro_pass_wait_timeouts() == 0


@pytest.mark.parametrize("n", [32, 512])
def test_half_paired_steady_kernel_matches_oracle(n):
    """The half-paired steady pass (tune bit 256; decimation in frequency inside the
    thread) agrees with the oracle and the one-line kernel to float32 rounding; at
    512^2 its TMA column variant (bit 2048) and its half-pair interleaved
    transmission tables (bit 16384) give the same bits as the plain variant."""
    import numpy as np
    from oracle import multislice_ref as R
    from tests.conftest import rel_l2
    from ptyrodactyl_b200.simulations import run_forward
    rng = np.random.default_rng(n + 1)
    s, p = 6, 3
    pot = rng.uniform(0, 40, (n, n, s))
    probe = R.make_probe(200.0, 25.0, (n, n), 30.0, defocus_ang=-20.0)
    dev = torch.device("cuda")
    slices = torch.as_tensor(pot, dtype=torch.float32, device=dev)
    modes = torch.as_tensor(probe[..., None].astype(np.complex64), device=dev)
    wt = torch.ones(1, device=dev)
    pos = rng.uniform(-2, 2, (p, 2))
    pos_d = torch.as_tensor(pos, dtype=torch.float64, device=dev)
    ref = run_forward(slices, 1.7, modes, wt, pos_d, 200.0, 0.3, 0.3, tune=3, lanes=1).cpu().numpy()
    want = R.stem_4d(pot, 1.7, 0.3, probe[..., None], [1.0], 0.3, 200.0, pos, 0.3, dtype=np.complex128)["data"]
    outs = {}
    for tune in (259, 771, 2307, 2819, 18691, 19203):
        got = run_forward(slices, 1.7, modes, wt, pos_d, 200.0, 0.3, 0.3, tune=tune, lanes=1).cpu().numpy()
        assert rel_l2(got, want) < 1e-4
        assert rel_l2(got, ref) < 2e-6
        outs[tune] = got
    assert np.array_equal(outs[2307], outs[259]) and np.array_equal(outs[2819], outs[771])
    assert np.array_equal(outs[18691], outs[259]) and np.array_equal(outs[19203], outs[771])
    torch.cuda.synchronize()
    assert pb._lib.load().ptyro_pass_wait_timeouts() == 0


def test_ragged_batches_and_lanes_at_256_match_one_line_kernel():
    """At 256^2 the default launch variant (TMA column blocks with tensor maps encoded
    per batch size, paired first/last passes, interleaved transmission tables) gives
    the one-line kernel's bits with a ragged last batch and several lanes."""
    import numpy as np
    from oracle import multislice_ref as R
    from ptyrodactyl_b200.simulations import default_tune, run_forward
    rng = np.random.default_rng(256)
    n, s, p = 256, 6, 37
    dev = torch.device("cuda")
    slices = torch.as_tensor(rng.uniform(0, 40, (n, n, s)), dtype=torch.float32, device=dev)
    probe = R.make_probe(200.0, 25.0, (n, n), 30.0, defocus_ang=-20.0)
    modes = torch.as_tensor(probe[..., None].astype(np.complex64), device=dev)
    wt = torch.ones(1, device=dev)
    pos = torch.as_tensor(rng.uniform(-2, 2, (p, 2)), dtype=torch.float64, device=dev)
    ref = run_forward(slices, 1.7, modes, wt, pos, 200.0, 0.3, 0.3, tune=3, batch=8, lanes=1)
    for lanes in (1, 3):
        got = run_forward(slices, 1.7, modes, wt, pos, 200.0, 0.3, 0.3, tune=default_tune(n), batch=8, lanes=lanes)
        assert torch.equal(got, ref), lanes
    torch.cuda.synchronize()
    assert pb._lib.load().ptyro_pass_wait_timeouts() == 0
