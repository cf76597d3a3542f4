"""CPU checks of the proposal network's oracle (float64 restatement): its
backward against central finite differences of its own forward, the bf16
rounding against torch's, and the VSBP blob format."""
import numpy as np
import pytest

import pnet_oracle as P


def _params(seed):
    bits, f32 = P.init_params(seed)
    p = P.unpack(bits, f32)
    rng = np.random.default_rng(seed + 1)
    for k in ("b1", "b2", "b3", "b4"):
        p[k] = rng.normal(0.05, 0.05, 32)
    p["bfc"] = rng.normal(0, 0.1, 3)
    return p


def test_bf16_round_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.normal(0, 1, 5000), rng.normal(0, 1e-3, 500), [0.0, -0.0, 1.0, 255.0]])
    x = x.astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(P.bf16_round(x).astype(np.float32), ref)


def test_backward_matches_finite_differences():
    """gradient of sum(out * dout) for every parameter tensor, float64 with
    the storage rounding off, against central differences"""
    rng = np.random.default_rng(3)
    p = _params(3)
    x = rng.normal(0, 1, (2, 32, 32, 2))
    dout = rng.normal(0, 1, (2, 3))
    acts, out = P.forward(p, x, rounding=False)
    gb, gf = P.backward(p, x, acts, dout)

    def f(q):
        return float((P.forward(q, x, rounding=False)[1] * dout).sum())

    offs = {"W1": 0, "W2": P.N_W1, "W3": P.N_W1 + P.N_W, "W4": P.N_W1 + 2 * P.N_W,
            "Wfc": P.N_W1 + 3 * P.N_W}
    eps = 1e-6
    for name, off in offs.items():
        flat = p[name].ravel()
        cand = np.arange(flat.size)
        if name == "W1":
            cand = cand[(cand % 32) < 18]
        for j in rng.choice(cand, 6, replace=False):
            q = {k: v.copy() for k, v in p.items()}
            q[name].ravel()[j] += eps
            fp = f(q)
            q[name].ravel()[j] -= 2 * eps
            fm = f(q)
            num = (fp - fm) / (2 * eps)
            assert abs(num - gb[off + j]) <= 1e-5 * max(1.0, abs(num)), (name, j, num, gb[off + j])
    for bi, name in enumerate(("b1", "b2", "b3", "b4", "bfc")):
        n = 3 if name == "bfc" else 32
        for j in rng.choice(n, 3, replace=False):
            q = {k: v.copy() for k, v in p.items()}
            q[name][j] += eps
            fp = f(q)
            q[name][j] -= 2 * eps
            fm = f(q)
            num = (fp - fm) / (2 * eps)
            assert abs(num - gf[32 * bi + j]) <= 1e-5 * max(1.0, abs(num)), (name, j)


def test_blob_roundtrip():
    from vidstab_b200 import pnet
    bits, f32 = P.init_params(1)
    blob = pnet.pack_blob(bits, f32, 4.0, 2.0, -1.5, 33.0)
    assert len(blob) == 32 + pnet.PARAM_BYTES
    b2, f2, meta = pnet.unpack_blob(blob)
    assert np.array_equal(b2, bits) and np.array_equal(f2, f32)
    assert meta == {"scale": 4.0, "radius": 2.0, "conf_min": -1.5, "match_bound": 33.0}
    with pytest.raises(ValueError):
        pnet.unpack_blob(b"XXXX" + blob[4:])
