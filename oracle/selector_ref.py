"""CPU restatement of the per-block format selection -- TEST INFRASTRUCTURE ONLY.

* candidate payloads of a 2048-value block (the bytes the reference's
  morph_batch writes for each candidate, via the C oracle);
* the sampled statistics the learned selector reads (engine's k_sel_features);
* the MLP's forward pass and gradients in float64 with the GPU's BF16
  rounding points (weights, and every matrix-product input), to check the
  tensor-core training kernels;
* the blockwise container layout (blockwise_individual.h:169-311).
"""
from __future__ import annotations

import numpy as np

from . import DELTA_DVBP, DYNAMIC_VBP, FOR_DVBP, RLE, STATIC_VBP, Oracle

BLOCK = 2048
CODES = {0: None, 1: 65, 2: 67, 3: 69, 4: 71}


def eff_bw(v: np.ndarray) -> np.ndarray:
    v = np.asarray(v, dtype=np.uint64) | np.uint64(1)
    out = np.zeros(v.shape, dtype=np.int64)
    for b in range(64):
        out = np.where(v >> np.uint64(b) != 0, b + 1, out)
    return out


def candidate_payload(orc: Oracle, x: np.ndarray, c: int):
    """(code, payload bytes) of one block in candidate c."""
    x = np.ascontiguousarray(x, dtype=np.uint64)
    assert len(x) == BLOCK
    if c == 0:
        bw = int(eff_bw(np.bitwise_or.reduce(x)).item())
        return bw, _pack(orc, STATIC_VBP, bw, x)
    fmt = {1: DYNAMIC_VBP, 2: DELTA_DVBP, 3: FOR_DVBP, 4: RLE}[c]
    return CODES[c], _pack(orc, fmt, 0, x)


def _pack(orc: Oracle, fmt: int, bw: int, x: np.ndarray) -> np.ndarray:
    import ctypes as C
    out = np.zeros(16 * BLOCK + 1024, dtype=np.uint8)
    if fmt == RLE:
        n = orc.lib.orc_rle_pack(x.ctypes.data_as(C.POINTER(C.c_uint64)), C.c_uint64(BLOCK),
                                 out.ctypes.data_as(C.POINTER(C.c_uint8)))
    else:
        orc.lib.orc_batch_pack.restype = C.c_uint64
        n = orc.lib.orc_batch_pack(C.c_int(fmt), C.c_uint(bw), x.ctypes.data_as(C.POINTER(C.c_uint64)),
                                   C.c_uint64(BLOCK), out.ctypes.data_as(C.POINTER(C.c_uint8)))
    return out[:n].copy()


def mask_for_header(payload: np.ndarray, c: int) -> np.ndarray:
    """for+dvbp of one block: header words after the end marker are not
    written by the reference (for.h:214-220)."""
    p = payload.copy()
    if c == 3:
        p[24:64] = 0
    return p


def payload_size(data: np.ndarray, pay: int, c: int, code: int) -> int:
    """Bytes of a block's payload at `pay` in candidate c, read from its
    headers: static_vbp 256 bw; dynamic_vbp one 64-B page header with four
    widths; delta+dvbp two such pages of two blocks; for+dvbp a 64-B header of
    references and then two pages (rle: 16 B per run, runs not recorded)."""
    if c == 0:
        return 256 * code
    if c == 1:
        return 64 + 64 * int(data[pay:pay + 4].astype(np.int64).sum())
    if c in (2, 3):
        p = pay + (64 if c == 3 else 0)
        for _ in range(2):
            p += 64 + 64 * int(data[p:p + 2].astype(np.int64).sum())
        return p - pay
    raise ValueError("rle payloads carry no size header")


def mask_container(data: np.ndarray, choice) -> np.ndarray:
    """A blockwise_individual_f container's bytes with the padding after every
    code byte and for_f's never-written header words zeroed: the reference
    leaves both unwritten (blockwise_individual.h:189-196, for.h:214-220).
    Blocks must not be rle (its payload has no size header)."""
    x = np.array(data, dtype=np.uint8, copy=True)
    pos = 0
    for c in choice:
        code_end = pos + 1
        pay = (code_end + 63) // 64 * 64
        x[code_end:pay] = 0
        if int(c) == 3:
            x[pay + 24:pay + 64] = 0
        pos = pay + payload_size(x, pay, int(c), int(x[pos]))
    if pos != len(x):
        raise ValueError(f"container walk ends at {pos}, not at {len(x)}")
    return x


def shared_code(ref_code: int) -> int:
    """The reference exhaustive selector's pick in the GPU's code space:
    uncompr (chosen when a block needs all 64 bits) is static_vbp<64> there
    (identical bytes); group_simple picks (66, 68, 70) have no GPU
    counterpart and map to -1."""
    if ref_code == 0:
        return 64
    return ref_code if ref_code <= 65 or ref_code in (67, 69) else -1


def container_positions(sizes: np.ndarray):
    """(code byte offset, payload offset) per block and the total size."""
    q = np.zeros(len(sizes), dtype=np.int64)
    if len(sizes) > 1:
        q[1:] = np.cumsum(64 + (sizes[:-1] // 64) * 64)
    code = q.copy()
    code[1:] += sizes[:-1] % 64
    total = int(q[-1] + 64 + sizes[-1]) if len(sizes) else 0
    return code, q + 64, total


def features(x: np.ndarray) -> np.ndarray:
    """The 32 sampled statistics (rows 512c .. 512c+63 of each quarter)."""
    x = np.asarray(x, dtype=np.uint64)
    hv = np.zeros(8)
    hd = np.zeros(8)
    vb, db, negs, zds, heads = [], [], 0, 0, 0
    cmax, cdmax = [0] * 4, [0] * 4
    samples = []
    nd = 0
    for c in range(4):
        ch = x[512 * c: 512 * c + 64]
        samples.append(ch)
        bws = eff_bw(ch)
        for b in bws:
            hv[(b - 1) >> 3] += 1
        vb.extend(bws.tolist())
        cmax[c] = int(bws.max())
        d = (ch[8:] - ch[:-8]).astype(np.uint64)
        dbw = eff_bw(d)
        for b in dbw:
            hd[(b - 1) >> 3] += 1
        db.extend(dbw.tolist())
        cdmax[c] = int(dbw.max())
        negs += int((d.view(np.int64) < 0).sum())
        zds += int((d == 0).sum())
        nd += len(d)
        heads += int((ch[1:] != ch[:-1]).sum())
    s = np.concatenate(samples)
    f = np.zeros(32, dtype=np.float64)
    f[0:8] = hv / 256.0
    f[8:16] = hd / nd
    f[16] = max(vb) / 64.0
    f[17] = min(vb) / 64.0
    f[18] = eff_bw(np.array([int(s.max()) - int(s.min())], dtype=np.uint64))[0] / 64.0
    f[19] = max(db) / 64.0
    f[20] = negs / nd
    f[21] = heads / 252.0
    f[22] = zds / nd
    f[23] = sum(vb) / (256 * 64.0)
    f[24:28] = np.array(cmax) / 64.0
    f[28:32] = np.array(cdmax) / 64.0
    return f.astype(np.float32)


# ---------------------------------------------------------------------------
# MLP 32 -> 64 -> 64 -> 5 with ReLU, mean squared error on log2 sizes
# ---------------------------------------------------------------------------
IN, H, OUT = 32, 64, 5
LAYOUT = [("W1", (H, IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (OUT, H)), ("b3", (OUT,))]


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even) and back."""
    u = np.asarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(params: np.ndarray):
    out, o = {}, 0
    for name, shape in LAYOUT:
        n = int(np.prod(shape))
        out[name] = params[o: o + n].reshape(shape).astype(np.float64)
        o += n
    return out


def forward(params: np.ndarray, feats: np.ndarray) -> np.ndarray:
    """Predicted log2 sizes, with the GPU's rounding points (see below)."""
    w = unpack(bf16(params))
    r = lambda a: bf16(a.astype(np.float32)).astype(np.float64)  # noqa: E731
    h1 = r(np.maximum(r(feats) @ w["W1"].T + w["b1"], 0))
    h2 = r(np.maximum(h1 @ w["W2"].T + w["b2"], 0))
    return h2 @ w["W3"].T + w["b3"]


def loss_and_grads(params: np.ndarray, feats: np.ndarray, sizes: np.ndarray):
    """Loss and gradient (parameter order) for a batch, float64 arithmetic
    with the GPU's rounding points: BF16 weights; features, hidden
    activations and backward deltas rounded to BF16 where they enter a matrix
    product; biases, ReLU masks and bias gradients on the unrounded values."""
    w = unpack(bf16(params))
    r = lambda a: bf16(a.astype(np.float32)).astype(np.float64)  # noqa: E731
    x = r(feats)
    y = np.log2(sizes.astype(np.float64))
    z1 = x @ w["W1"].T + w["b1"]
    h1 = r(np.maximum(z1, 0))
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = r(np.maximum(z2, 0))
    o = h2 @ w["W3"].T + w["b3"]
    e = o - y
    B = len(x)
    loss = (e ** 2).sum() / (B * OUT)
    do = 2 * e / (B * OUT)
    g = {"W3": r(do).T @ h2, "b3": do.sum(0)}
    d2 = (r(do) @ w["W3"]) * (z2 > 0)
    g["W2"], g["b2"] = r(d2).T @ h1, d2.sum(0)
    d1 = (r(d2) @ w["W2"]) * (z1 > 0)
    g["W1"], g["b1"] = r(d1).T @ x, d1.sum(0)
    flat = np.concatenate([g[name].ravel() for name, _ in LAYOUT])
    return loss, flat
