"""The learned prefilter's device code against plain PyTorch fp32 references.

* the tensor-core GEMM (tcgen05.mma, bf16 operands, fp32 accumulation) against
  torch's fp32 matmul of the same bf16 values, for every shape and epilogue the
  network uses (bias, ReLU, ReLU-backward mask, bf16 row-major and transposed
  stores, fp32 store);
* the network's forward pass against a torch restatement that rounds the
  activations to bf16 between layers as the device does;
* one optimizer step: the first Adam step moves every parameter by -lr*sign(grad)
  wherever the gradient is not tiny, so the signs of the device's parameter
  deltas must equal the signs of torch autograd's gradients of the same loss;
* the candidate features against the numpy restatement in tests/pf_ref.py.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from protlocus_b200 import lib as L

pytestmark = pytest.mark.gpu

DEV = "cuda"


def bf(x):
    return x.to(torch.bfloat16)


def gemm(A, B, *, n_tile=None, bias=None, relu=False, mask=None, want=("C", "CT", "Cf")):
    M, K = A.shape
    N = B.shape[0]
    n_tile = n_tile or min(N, 256)
    Cm = torch.zeros(M, N, dtype=torch.bfloat16, device=DEV) if "C" in want else None
    CT = torch.zeros(N, M, dtype=torch.bfloat16, device=DEV) if "CT" in want else None
    Cf = torch.zeros(M, N, dtype=torch.float32, device=DEV) if "Cf" in want else None
    err = torch.zeros(1, dtype=torch.int32, device=DEV)
    ptr = (lambda t: t.data_ptr() if t is not None else None)
    ok = L.load().pl_pf_gemm(0, A.data_ptr(), K, B.data_ptr(), K, M, N, K, n_tile, ptr(bias), int(relu), ptr(mask),
                             N, ptr(Cm), N, ptr(CT), M, ptr(Cf), N, err.data_ptr(), None)
    assert ok, L.error()
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return Cm, CT, Cf


@pytest.mark.parametrize("M,N,K,n_tile", [(128, 16, 64, 16), (256, 256, 576, 256), (512, 576, 256, 192),
                                          (256, 128, 4096, 128), (384, 64, 128, 32)])
def test_gemm_matches_torch(M, N, K, n_tile):
    g = torch.Generator(device="cpu").manual_seed(M * 7 + N * 3 + K)
    A = bf(torch.randn(M, K, generator=g)).to(DEV)
    B = bf(torch.randn(N, K, generator=g) / K ** 0.5).to(DEV)
    bias = torch.randn(N, generator=g).to(DEV)
    mask = bf(torch.randn(M, N, generator=g)).to(DEV)
    ref = A.float() @ B.float().T
    _, _, Cf = gemm(A, B, n_tile=n_tile, want=("Cf",))
    tol = 1e-3 * ref.abs().max().item() + 1e-4
    assert (Cf - ref).abs().max().item() <= tol
    Cm, CT, Cf2 = gemm(A, B, n_tile=n_tile, bias=bias, relu=True, mask=mask)
    want = torch.relu(ref + bias) * (mask.float() > 0)
    assert (Cf2 - want).abs().max().item() <= tol
    assert (Cm.float() - want).abs().max().item() <= tol + 8e-3 * want.abs().max().item()
    assert torch.equal(CT, Cm.T)


def _model(seed=3, hidden=256):
    lib = L.load()
    h = lib.pl_pf_model_create(0, 576, hidden, seed)
    assert h, L.error()
    n = lib.pl_pf_model_size(h)
    p = np.zeros(n, dtype=np.float32)
    assert lib.pl_pf_model_get(h, p.ctypes.data, n)
    return h, p


def _unpack(p, hidden=256, fdim=576):
    dims = [(hidden, fdim), (hidden, hidden), (hidden, hidden), (16, hidden)]
    out, off = [], 0
    for o, i in dims:
        W = p[off:off + o * i].reshape(o, i)
        off += o * i
        b = p[off:off + o]
        off += o
        out.append((torch.from_numpy(W.copy()), torch.from_numpy(b.copy())))
    return out


def _torch_forward(layers, X, round_acts=True):
    h = X
    for li, (W, b) in enumerate(layers):
        z = h @ bf(W).float().T + b
        if li < 3:
            h = torch.relu(z)
            if round_acts:
                h = bf(h).float()
        else:
            h = z
    return h


def test_forward_matches_torch():
    lib = L.load()
    h, p = _model()
    try:
        n = 300
        npad = 384
        g = torch.Generator().manual_seed(5)
        X = bf(torch.rand(npad, 576, generator=g))
        X[n:] = 0
        Xd = X.to(DEV)
        out = torch.zeros(npad, 16, dtype=torch.float32, device=DEV)
        assert lib.pl_pf_predict(h, Xd.data_ptr(), n, out.data_ptr(), None), L.error()
        torch.cuda.synchronize()
        ref = _torch_forward(_unpack(p), X.float())
        got = out.cpu()[:n]
        scale = ref[:n, :3].abs().max().item()
        assert (got[:, :3] - ref[:n, :3]).abs().max().item() <= 2e-2 * scale + 1e-3
    finally:
        lib.pl_pf_model_destroy(h)


def test_first_adam_step_follows_gradient_signs():
    lib = L.load()
    h, p0 = _model(seed=9)
    try:
        B = 256
        g = torch.Generator().manual_seed(11)
        X = bf(torch.rand(B, 576, generator=g))
        y = (torch.rand(B, generator=g) < 0.3).float()
        ts, te = torch.rand(B, generator=g) * 0.5, 0.5 + torch.rand(B, generator=g) * 0.5
        T = torch.stack([y, ts, te, y], 1).float()
        perm = torch.arange(B, dtype=torch.int32)
        Xd, Td, Pd = X.to(DEV), T.to(DEV), perm.to(DEV)
        lr = 1e-4
        loss = np.zeros(1, dtype=np.float32)
        assert lib.pl_pf_train(h, Xd.data_ptr(), Td.data_ptr(), Pd.data_ptr(), B, B, 1, lr, 2.0, 1.0,
                               loss.ctypes.data, None), L.error()
        n = p0.size
        p1 = np.zeros(n, dtype=np.float32)
        assert lib.pl_pf_model_get(h, p1.ctypes.data, n)
        # torch: the same loss on the same bf16 weights, activations rounded as on the device
        layers = [(bf(W).float().requires_grad_(), b.clone().requires_grad_()) for W, b in _unpack(p0)]
        hdn = X.float()
        for li, (W, b) in enumerate(layers):
            z = hdn @ W.T + b
            hdn = torch.relu(z) if li < 3 else z
        z0, s, e = hdn[:, 0], hdn[:, 1], hdn[:, 2]
        cw = torch.where(y > 0.5, 2.0, 1.0)
        bce = cw * (torch.clamp(z0, min=0) - z0 * y + torch.log1p(torch.exp(-z0.abs())))

        def hub(d):
            return torch.where(d.abs() < 0.05, d * d / 0.1, d.abs() - 0.025)
        tot = (bce + 1.0 * y * (hub(s - ts) + hub(e - te))).mean()
        assert abs(tot.item() - float(loss[0])) <= 2e-2 * abs(tot.item()) + 1e-3
        tot.backward()
        grads = []
        for W, b in layers:
            grads += [W.grad.reshape(-1), b.grad.reshape(-1)]
        gr = torch.cat(grads).numpy()
        d = p1 - p0
        big = np.abs(gr) > 0.02 * np.abs(gr).max()
        assert big.sum() > 300
        agree = (np.sign(d[big]) == -np.sign(gr[big])).mean()
        assert agree > 0.98, agree
    finally:
        lib.pl_pf_model_destroy(h)


def test_features_match_restatement():
    import pf_ref
    from protlocus_b200 import prefilter as P
    from protlocus_b200.abi import make_tables
    cand = P.make_candidates(3, n_prot=6, win_max=9000)
    eng = L.Engine(0)
    try:
        pipe = P.Pipeline(eng, cand)
        feats, chain = pipe.features()
        torch.cuda.synchronize()
        F = feats.float().cpu().numpy()
        ch = chain.cpu().numpy()
        nt4, aa20, codon = make_tables()
        n_chain = 0
        for q, j in enumerate(cand["jobs"]):
            nt = cand["nt"][j["nt_off"]: j["nt_off"] + j["nl"]].tobytes()
            aa = cand["aa"][j["aa_off"]: j["aa_off"] + j["al"]].tobytes()
            want, wchain, na, length = pf_ref.features(nt, aa, nt4, aa20, codon)
            assert np.array_equal(F[q, :512], want[:512]), q
            assert list(ch[q]) == wchain, (q, list(ch[q]), wchain)
            # scalars: within one bf16 ulp (device log2f may differ from numpy's by an ulp)
            assert np.allclose(F[q, 512:], want[512:], rtol=2 ** -7, atol=1e-6), (q, F[q, 512:532], want[512:532])
            n_chain += length >= 10
        assert n_chain >= 6  # the true windows chain
        assert not F[len(cand["jobs"]):].any()
    finally:
        eng.close()


def test_learned_path_small():
    """A few hundred candidates end to end: labels from the plain DP, a short training
    run lowers the loss, and the learned path with a permissive threshold reports every
    candidate the plain path passes."""
    from protlocus_b200 import prefilter as P
    eng = L.Engine(0)
    model = P.PrefilterModel(0, seed=2)
    try:
        data = P.build_set(eng, [11, 12], n_prot=64, workers=1)
        assert data["n"] == 2 * 64 * 8 and data["labels"].sum() >= 100
        losses = P.train(model, data, epochs=40, batch=256, lr=2e-3)
        assert losses[-10:].mean() < 0.7 * losses[:10].mean(), (losses[:10], losses[-10:])
        cand = P.make_candidates(13, n_prot=64)
        pipe = P.Pipeline(eng, cand)
        plain, _ = pipe.plain()
        passed, stats = pipe.learned(model, tau=1e-4, margin=400, rel=0.2)
        assert stats["kept"] <= pipe.n
        m = P.path_metrics(pipe, plain, passed)
        assert m["plain_loci"] >= 40 and m["locus_recall"] >= 0.97, m
    finally:
        model.close()
        eng.close()


def test_shipped_model_locus_recall():
    """The shipped model and thresholds on 1024 proteins of the held-out seed 65 (8192
    candidates): the learned path reports at least 99.5 % of the loci the plain path
    reports, with every alignment from the exact DP."""
    import os
    from protlocus_b200 import prefilter as P
    path = os.path.join(os.path.dirname(P.__file__), "data", "prefilter.npz")
    eng = L.Engine(0)
    model, meta = P.load_model(path, 0)
    try:
        assert "1-64" in str(meta["train_seeds"]) and int(meta["val_seed"]) not in range(1, 66)
        cand = P.make_candidates(65, n_prot=1024)
        pipe = P.Pipeline(eng, cand)
        plain, _ = pipe.plain()
        passed, stats = pipe.learned(model, float(meta["tau"]), int(meta["margin"]), 0.0, float(meta["tau_fb"]))
        m = P.path_metrics(pipe, plain, passed)
        print(m, stats)
        assert m["plain_loci"] >= 500 and m["locus_recall"] >= 0.995, m
        assert stats["cells_tight"] < 0.2 * int(((cand["jobs"]["nl"].astype(np.int64) - 2) * cand["jobs"]["al"]).sum())
    finally:
        model.close()
        eng.close()
