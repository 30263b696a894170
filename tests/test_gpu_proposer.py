"""The learned proposer's CUDA kernels against the FP64 oracle
(oracle/proposer_oracle.py): forward-model features, features from a
resident G, the winner-takes-all loss, and the MLP's outputs and gradients;
a short training run that must cut the validation error; what the trained
network gains over the plain sweep; and a held-out check of the training
data against fully simulated scans."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest
import torch

from oracle import proposer_oracle as po
from oracle import ssb_oracle as so
from quantem.gpu_b200 import _lib, proposer as pr
from quantem.gpu_b200.synthetic import draw_aberrations

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _host_csr(lat):
    return lat.off.cpu().numpy(), lat.idx.cpu().numpy(), lat.w.cpu().numpy()


def test_synth_features_match_oracle():
    tl = pr.TrainingLattice(DEV)
    rng = np.random.default_rng(2)
    ab = draw_aberrations(rng, 3)
    nq = len(pr.Q_UNITS)
    phi = np.zeros((3, nq, 2, 2), np.float32)
    phi[:, :, 0, 0] = 1.0  # unit phase-object spectrum, no amplitude part
    sig = np.zeros((3, nq), np.float32)
    lat = tl.lattice
    scratch = torch.empty(3 * nq * lat.n_bf, device=DEV)
    out = torch.empty((3, pr.N_IN), device=DEV)
    ab_d, phi_d, sig_d = (torch.as_tensor(a, device=DEV) for a in (ab, phi, sig))
    _lib.check(_lib.load().qssb_synth_features(
        _ptr(tl.geom), lat.n_bf, _ptr(tl.q_vec), nq, _ptr(ab_d), _ptr(phi_d), _ptr(sig_d), 3,
        ctypes.byref(tl.cal), 0, _ptr(lat.off), _ptr(lat.idx), _ptr(lat.w), pr.GRID * pr.GRID,
        _ptr(scratch), _ptr(out), None, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    got = out.cpu().numpy().reshape(3, nq, -1)
    g = tl.geom.cpu().numpy().astype(np.float64)
    geo = so.Geometry(g[0], g[1], g[2], g[3], g[4], g[5], np.zeros(1), np.zeros(1), tl.wavelength,
                      pr.TRAIN_SEMIANGLE_MRAD * 1e-3, pr.TRAIN_DET_SAMPLING_MRAD * 1e-3,
                      pr.TRAIN_DET_SAMPLING_MRAD * 1e-3)
    off, idx, w = _host_csr(lat)
    qv = tl.q_vec.cpu().numpy().astype(np.float64)
    for s in range(3):
        a = so.Aberrations(*map(float, ab[s]))
        vals = np.stack([np.abs(po.gamma(qv[q, 0], qv[q, 1], g[0] + g[6], g[1] + g[7], g[2], g[3],
                                         g[4], g[5], a, geo)) for q in range(nq)])
        want = po.resample(vals, off, idx, w)
        np.testing.assert_allclose(got[s], want, atol=2e-3)


def test_backend_features_match_oracle():
    from quantem.gpu_b200 import B200SSBBackend
    from quantem.gpu_b200.synthetic import CONFIGS, generate

    spec = CONFIGS["plain_128x128_det128"]
    be = B200SSBBackend(generate(spec, DEV).counts, semiangle=spec.semiangle_mrad,
                        scan_sampling=spec.scan_step_A, det_sampling=spec.det_sampling_mrad,
                        voltage_kV=spec.voltage_kV, device=DEV)
    got = pr.backend_features(be).float().cpu().numpy().reshape(len(pr.Q_UNITS), -1)
    g = be.G_qk.cpu().numpy()
    n = be.scan_shape[0]
    vals = []
    for m, k in pr.Q_UNITS * 2:
        r, c = m % n, k % n
        if c > n // 2:
            r, c = (n - r) % n, n - c
        vals.append(np.abs(g[:, r, c]).astype(np.float64))
    off, idx, w = _host_csr(be._proposer_lattice)
    want = po.resample(np.stack(vals), off, idx, w)
    np.testing.assert_allclose(got, want, rtol=1e-2, atol=1e-2)  # BF16 output


def test_mse_heads_matches_oracle():
    """``qssb_mse_heads`` on given FP32 outputs: loss, gradient and winners
    equal the FP64 oracle's (one head reduces to the plain MSE)."""
    rng = np.random.default_rng(11)
    m, n_out, heads, ld = 64, 4, 4, 16
    y = torch.as_tensor(rng.normal(size=(m, ld)).astype(np.float32), device=DEV)
    t = torch.as_tensor(rng.normal(size=(m, n_out)).astype(np.float32), device=DEV)
    w = torch.as_tensor(np.array([1.0, 1.0, 1.0, 0.1], np.float32), device=DEV)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for h, n_sel, eps in ((4, 3, 0.05), (4, 4, 0.0), (1, 4, 0.0)):
        dy = torch.full((m, ld), 7.0, device=DEV)
        loss = torch.empty(1, device=DEV)
        win = torch.empty(m, dtype=torch.int32, device=DEV)
        _lib.check(_lib.load().qssb_mse_heads(_ptr(y), _ptr(t), m, n_out, h, ld, _ptr(w), n_sel,
                                              ctypes.c_float(eps), _ptr(dy), _ptr(loss), _ptr(win),
                                              stream))
        l_ref, dy_ref, win_ref = po.heads_loss_and_grad(y.cpu().numpy(), t.cpu().numpy(), n_out, h,
                                                        w.cpu().numpy(), n_sel, eps)
        np.testing.assert_array_equal(win.cpu().numpy(), win_ref)
        np.testing.assert_allclose(dy.cpu().numpy(), dy_ref, rtol=1e-5, atol=1e-9)
        assert abs(loss.item() - l_ref) <= 1e-6 * l_ref
    bad = _lib.load().qssb_mse_heads(_ptr(y), _ptr(t), m, n_out, 5, ld, None, 3,
                                     ctypes.c_float(0.0), _ptr(dy), None, None, stream)
    assert bad != 0  # 5 heads x 4 outputs do not fit 16 columns


def test_mlp_outputs_and_gradients_match_oracle():
    """Forward outputs and every gradient of the winner-takes-all training
    step against the FP64 oracle. Row r's target lies within 0.01 of head
    r mod 4 in (C1, A1), which select the winner, so that the winners do not
    hang on BF16 rounding, and is drawn freely in C3, which then carries most
    of the loss."""
    mlp = pr.MLP(DEV, seed=3)
    rng = np.random.default_rng(4)
    m = 32
    x = torch.as_tensor(rng.uniform(0, 2, size=(m, pr.N_IN)).astype(np.float32), device=DEV).to(torch.bfloat16)
    ws = [w.float().cpu().numpy().astype(np.float64) for w in mlp.w_bf]
    bs = [b.cpu().numpy().astype(np.float64) for b in mlp.b]
    y = mlp.forward(x).cpu().numpy()
    heads = y[:, :pr.HEADS * pr.N_OUT].reshape(m, pr.HEADS, pr.N_OUT)
    t_np = heads[np.arange(m), np.arange(m) % pr.HEADS] + 0.01 * rng.normal(size=(m, pr.N_OUT))
    t_np[:, 3] = rng.normal(size=m)
    t_np = t_np.astype(np.float32)
    t = torch.as_tensor(t_np, device=DEV)
    loss_ref, y_ref, dws, dbs = po.mlp_loss_and_grads(x.float().cpu().numpy(), ws, bs, t_np,
                                                       pr.N_OUT, pr.HEADS, pr.OUT_WEIGHT, 3,
                                                       pr.WTA_EPS)
    np.testing.assert_allclose(y, y_ref, rtol=2e-2, atol=2e-2)
    loss = mlp.backward_and_step(t, lr=0.0).item()
    bufs = mlp._buf(m)
    np.testing.assert_array_equal(bufs["winner"].cpu().numpy(), np.arange(m) % pr.HEADS)
    assert abs(loss - loss_ref) <= 2e-2 * loss_ref
    for i in range(4):
        for got, want in ((bufs["gw"][i].cpu().numpy(), dws[i]), (bufs["gb"][i].cpu().numpy(), dbs[i])):
            rel = np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-30)
            assert rel <= 3e-2, (i, rel)


def test_device_schedule_matches_host_adam():
    """``qssb_adam_schedule`` + ``qssb_adam_dev`` give the update ``qssb_adam``
    gives with the host's cosine learning rate and bias corrections."""
    import math

    lib = _lib.load()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    g = torch.Generator(device=DEV).manual_seed(9)
    n, total, first, lr = 4096, 50, 3, 1e-3
    w = torch.randn(n, generator=g, device=DEV)
    grad = torch.randn(n, generator=g, device=DEV)
    m0 = 0.1 * torch.randn(n, generator=g, device=DEV)
    v0 = torch.rand(n, generator=g, device=DEV)
    hyper = torch.zeros(4, device=DEV)
    step = torch.full((1,), first + 6, dtype=torch.int32, device=DEV)  # 7th step of the run
    _lib.check(lib.qssb_adam_schedule(_ptr(hyper), _ptr(step), first, total, ctypes.c_float(lr),
                                      ctypes.c_float(0.9), ctypes.c_float(0.999), stream))
    t = first + 7
    assert int(step.item()) == t
    want_lr = lr * 0.5 * (1.0 + math.cos(math.pi * (t - 1 - first) / total))
    h = hyper.cpu().numpy()
    np.testing.assert_allclose(h[0], want_lr, rtol=1e-6)
    # 1 - powf(beta, t) in float32, as qssb_adam forms it: the float32 betas,
    # and a powf error of an ulp or two magnified by the cancellation
    b1, b2 = float(np.float32(0.9)), float(np.float32(0.999))
    np.testing.assert_allclose(h[1:3], [1 - b1 ** t, 1 - b2 ** t], rtol=3e-5)
    w1, m1, v1 = w.clone(), m0.clone(), v0.clone()
    w2, m2, v2 = w.clone(), m0.clone(), v0.clone()
    _lib.check(lib.qssb_adam_dev(_ptr(w1), _ptr(m1), _ptr(v1), _ptr(grad), n, _ptr(hyper),
                                 ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8),
                                 ctypes.c_float(1e-5), None, stream))
    _lib.check(lib.qssb_adam(_ptr(w2), _ptr(m2), _ptr(v2), _ptr(grad), n, ctypes.c_float(h[0]),
                             ctypes.c_float(0.9), ctypes.c_float(0.999), ctypes.c_float(1e-8),
                             ctypes.c_float(1e-5), t, None, stream))
    assert torch.equal(m1, m2) and torch.equal(v1, v2)
    torch.testing.assert_close(w1, w2, rtol=1e-6, atol=1e-9)


def test_graph_replayed_training_equals_eager_steps():
    """Training replayed from the captured step graph gives the same weights,
    bit for bit, as the same steps launched one by one."""
    a = pr.Proposer(DEV, seed=4)
    b = pr.Proposer(DEV, seed=4)
    ia = a.train(n_samples=2048, epochs=3, use_graph=True)
    ib = b.train(n_samples=2048, epochs=3, use_graph=False)
    assert ia["graph"] and not ib["graph"] and ia["steps"] == ib["steps"] == 3 * 8
    assert a.mlp.t == b.mlp.t == 24
    for wa, wb in zip(a.mlp.w + a.mlp.b, b.mlp.w + b.mlp.b):
        assert torch.equal(wa, wb)
    assert a.history == b.history


def test_short_training_cuts_validation_error():
    prop = pr.Proposer(DEV, seed=5)
    before = prop.validate(1024)["rmse_scaled"]
    prop.train(n_samples=20_000, epochs=10, batch=256, lr=1e-3)
    after = prop.validate(1024)["rmse_scaled"]
    assert after[0] < 0.5 * before[0], (before, after)       # C1
    assert np.mean(after[:3]) < 0.8 * np.mean(before[:3])     # C1 and A1


def test_learned_proposal_needs_fewer_evaluations_than_plain_sweep():
    """What the trained network gains: on weak-phase datasets (0.03 rad atoms,
    64^2 scans, 1e6 e per position) the proposal plus the 8-candidate
    refinement reaches a phase within 1e-4 rad RMS of the FP64 oracle at the
    true aberrations with at least 15x fewer SSB evaluations, in total over
    six cases, than the plain 64-candidate zoom sweep over the whole range;
    every learned fit reaches the target without the plain fallback."""
    from oracle import ssb_torch_fp64 as tf
    from quantem.gpu_b200 import B200SSBBackend
    from quantem.gpu_b200.synthetic import SyntheticSpec, generate

    prop = pr.Proposer(DEV, seed=0)
    prop.train(n_samples=50_000, epochs=40)
    rng = np.random.default_rng(77)
    plain_total = learned_total = 0
    for i in range(6):
        ab = draw_aberrations(rng, 1)[0]
        spec = SyntheticSpec(scan_shape=(64, 64), detector_shape=(64, 64),
                             det_sampling_mrad=20.0 / 12.0, dose=1e6, C10=float(ab[0]),
                             C12=float(ab[1]), phi12=float(ab[2]), C30=float(ab[3]),
                             atom_peak_rad=0.03, seed=100 + i)
        counts = generate(spec, DEV).counts
        be = B200SSBBackend(counts, semiangle=20.0, scan_sampling=0.5, det_sampling=20.0 / 12.0,
                            voltage_kV=300, device=DEV)
        padded = torch.as_tensor(so.pad_or_crop_scan(counts.cpu().numpy()), device=DEV)
        prep = tf.prepare(padded, voltage_kV=300, semiangle_mrad=20.0, scan_sampling=0.5,
                          det_sampling=20.0 / 12.0)
        truth = tf.reconstruct(prep, so.Aberrations(*map(float, ab)))[1].cpu().numpy()

        def ok(est):
            ph = be.object_and_phase(*map(float, est))[1].cpu().numpy()
            return float(np.sqrt(np.mean(so.wrapped_phase_error(ph, truth) ** 2))) <= 1e-4

        _, pe, _ = pr.zoom_search(be, None, (pr.BOX_HI - pr.BOX_LO) / 2, 64, 200, 0.75,
                                  np.random.default_rng(1), done=ok)
        best, le, _, fell_back = pr.learned_refine(be, pr.to_x(prop.propose(be)), done=ok)
        assert ok(best) and not fell_back, (i, le)
        plain_total += pe
        learned_total += le
    assert learned_total * 15 <= plain_total, (learned_total, plain_total)


def test_forward_model_features_match_simulated_scans():
    """Held-out check of the training data: for four aberration draws the
    network never saw, the forward model's 16 maps (all at reflections of the
    synthetic crystal; phase part only) match the maps measured from fully
    simulated 64^2 x 64^2 scans at 1e6 e per position (|FFT(probe x
    exp(i phi))|^2 per probe position, Poisson counts). Cosine similarity
    per map: on the
    configs' 0.3 rad objects every map >= 0.85 and the mean >= 0.97; on
    weak-phase (0.03 rad) objects, whose maps carry ten times less signal
    over the same counting noise, every map >= 0.8 and the mean >= 0.95.
    The lowest maps are those at the largest |Q| (24 / 32 A^-1), whose
    double-overlap lens is narrowest."""
    from quantem.gpu_b200 import B200SSBBackend
    from quantem.gpu_b200.synthetic import SyntheticSpec, generate

    lat = pr.TrainingLattice(DEV)
    for peak, lo, mean in ((0.3, 0.85, 0.97), (0.03, 0.8, 0.95)):
        rng = np.random.default_rng(2024)
        cos_all = []
        for i in range(4):
            ab = draw_aberrations(rng, 1)
            spec = SyntheticSpec(scan_shape=(64, 64), detector_shape=(64, 64),
                                 det_sampling_mrad=20.0 / 12.0, dose=1e6, C10=float(ab[0, 0]),
                                 C12=float(ab[0, 1]), phi12=float(ab[0, 2]), C30=float(ab[0, 3]),
                                 atom_peak_rad=peak, seed=500 + i)
            be = B200SSBBackend(generate(spec, DEV).counts, semiangle=20.0, scan_sampling=0.5,
                                det_sampling=20.0 / 12.0, voltage_kV=300, device=DEV)
            got = pr.backend_features(be).float().view(16, -1).cpu().numpy()
            want = lat.features(ab, np.random.default_rng(i), sigma=(1e-6, 1e-6),
                                informative=(16, 16), amplitude_contrast=(0.0, 0.0))
            want = want.float().view(16, -1).cpu().numpy()
            for q in range(16):
                a, b = got[q], want[q]
                cos_all.append(float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b))))
            be.close()
        assert min(cos_all) >= lo, (peak, cos_all)
        assert np.mean(cos_all) >= mean, (peak, np.mean(cos_all))
