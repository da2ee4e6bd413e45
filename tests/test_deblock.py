"""Deblocking of the reconstruction (the in-loop filter, crates/ironav-codec/src/h264/deblock.rs:232-695,
frame pictures, 4:2:0, as the encoder runs it before a picture becomes a reference, enc/mod.rs:650-655).

CPU: the oracle's tables against a fixture extracted from the reference (tests/golden/make_deblock_tables.py),
and the oracle against an independent pure-Python statement of the filter on small pictures, 8 and 10 bits.
GPU: the sm_100a kernel against the oracle, sample for sample, through the C ABI."""
from __future__ import annotations

import json
import os

import numpy as np
import pytest

from ironav_b200.inter import InterStage, IronavError
from ironav_b200.synth import dbk_encoder_slices as encoder_slices, dbk_planes as planes, dbk_records as records

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TABLES = json.load(open(os.path.join(GOLDEN, "deblock_tables.json")))


# ---- an independent statement of the filter (small pictures only) -----------------------------------------

def py_deblock(y, cb, cr, mbs, slices, mb_w, mb_h, bd):
    A, Bt, T, CQ = TABLES["alpha"], TABLES["beta"], TABLES["tc0"], TABLES["chroma_qp"]
    pl = [y.astype(np.int64), cb.astype(np.int64), cr.astype(np.int64)]
    maxv = (1 << bd) - 1

    def cqp(qp, off):
        v = min(max(qp + off, -6 * (bd - 8)), 51)
        return v if v < 30 else CQ[v - 30]

    def coded(m, bx, by):
        if m["t8x8"]:
            return any(m["nnz"][((by & 2) + dy) * 4 + (bx & 2) + dx] for dy in (0, 1) for dx in (0, 1))
        return m["nnz"][by * 4 + bx] > 0

    def far(a, b):
        return abs(int(a[0]) - int(b[0])) >= 4 or abs(int(a[1]) - int(b[1])) >= 4

    def differs(p, pb, q, qb):
        pi, qi = pb[1] * 4 + pb[0], qb[1] * 4 + qb[0]
        p8, q8 = (pb[1] // 2) * 2 + pb[0] // 2, (qb[1] // 2) * 2 + qb[0] // 2
        pr = [int(p["ref_id"][l][p8]) for l in (0, 1)]
        qr = [int(q["ref_id"][l][q8]) for l in (0, 1)]
        pm = [p["mv"][l][pi] for l in (0, 1)]
        qm = [q["mv"][l][qi] for l in (0, 1)]
        used_p = [l for l in (0, 1) if pr[l] >= 0]
        used_q = [l for l in (0, 1) if qr[l] >= 0]
        if len(used_p) != len(used_q):
            return True
        if len(used_p) == 1:
            a, b = used_p[0], used_q[0]
            return pr[a] != qr[b] or far(pm[a], qm[b])
        if sorted(pr) != sorted(qr):
            return True
        straight = far(pm[0], qm[0]) or far(pm[1], qm[1])
        crossed = far(pm[0], qm[1]) or far(pm[1], qm[0])
        if pr[0] != pr[1]:
            return straight if pr[0] == qr[0] else crossed
        return straight and crossed

    def uniform(m):
        return all((m["ref_idx"][l] == m["ref_idx"][l][0]).all() and (m["ref_id"][l] == m["ref_id"][l][0]).all()
                   and (m["mv"][l] == m["mv"][l][0]).all() for l in (0, 1))

    def line(v, b, tc0, alpha, beta, chroma):
        """v = [p3, p2, p1, p0, q0, q1, q2, q3] (chroma: p1, p0, q0, q1 at 2..5); the new values."""
        p3, p2, p1, p0, q0, q1, q2, q3 = v
        out = list(v)
        if abs(p0 - q0) >= alpha or abs(p1 - p0) >= beta or abs(q1 - q0) >= beta:
            return out
        if chroma:
            if b < 4:
                tc = tc0 + 1
                d = min(max((4 * (q0 - p0) + (p1 - q1) + 4) >> 3, -tc), tc)
                out[3], out[4] = min(max(p0 + d, 0), maxv), min(max(q0 - d, 0), maxv)
            else:
                out[3], out[4] = (2 * p1 + p0 + q1 + 2) >> 2, (2 * q1 + q0 + p1 + 2) >> 2
            return out
        ap, aq = abs(p2 - p0), abs(q2 - q0)
        if b < 4:
            tc = tc0 + (ap < beta) + (aq < beta)
            d = min(max((4 * (q0 - p0) + (p1 - q1) + 4) >> 3, -tc), tc)
            out[3], out[4] = min(max(p0 + d, 0), maxv), min(max(q0 - d, 0), maxv)
            if ap < beta:
                out[2] = p1 + min(max((p2 + ((p0 + q0 + 1) >> 1) - 2 * p1) >> 1, -tc0), tc0)
            if aq < beta:
                out[5] = q1 + min(max((q2 + ((p0 + q0 + 1) >> 1) - 2 * q1) >> 1, -tc0), tc0)
            return out
        small = abs(p0 - q0) < (alpha >> 2) + 2
        if ap < beta and small:
            out[3] = (p2 + 2 * p1 + 2 * p0 + 2 * q0 + q1 + 4) >> 3
            out[2] = (p2 + p1 + p0 + q0 + 2) >> 2
            out[1] = (2 * p3 + 3 * p2 + p1 + p0 + q0 + 4) >> 3
        else:
            out[3] = (2 * p1 + p0 + q1 + 2) >> 2
        if aq < beta and small:
            out[4] = (p1 + 2 * p0 + 2 * q0 + 2 * q1 + q2 + 4) >> 3
            out[5] = (p0 + q0 + q1 + q2 + 2) >> 2
            out[6] = (2 * q3 + 3 * q2 + q1 + q0 + p0 + 4) >> 3
        else:
            out[4] = (2 * q1 + q0 + p1 + 2) >> 2
        return out

    def filter_line(a, coords, b, tc0, alpha, beta, chroma, keep_p, keep_q):
        v = [int(a[c]) if c is not None else 0 for c in coords]
        new = line(v, b, tc0, alpha, beta, chroma)
        for k, c in enumerate(coords):
            if c is None or (k < 4 and keep_p) or (k >= 4 and keep_q):
                continue
            a[c] = new[k]

    for mby in range(mb_h):
        for mbx in range(mb_w):
            m = mbs[mby * mb_w + mbx]
            if m["slice"] == 0:
                continue
            sp = slices[m["slice"] - 1]
            if sp["disable_deblocking"] == 1:
                continue

            def usable(o):
                return o["slice"] != 0 and (sp["disable_deblocking"] == 0 or o["slice"] == m["slice"])

            nb = [mbs[mby * mb_w + mbx - 1] if mbx > 0 else m, mbs[(mby - 1) * mb_w + mbx] if mby > 0 else m]
            ok = [mbx > 0 and usable(nb[0]), mby > 0 and usable(nb[1])]
            still = bool(m["inter"]) and uniform(m) and not m["nnz"].any()
            bs = np.zeros((2, 4, 4), dtype=int)
            for d in (0, 1):
                for e in range(4):
                    if e > 0 and still:
                        continue
                    o = nb[d] if e == 0 else m
                    for i in range(4):
                        if not m["inter"] or not o["inter"]:
                            bs[d, e, i] = 4 if e == 0 else 3
                            continue
                        q = (e, i) if d == 0 else (i, e)
                        pe = 3 if e == 0 else e - 1
                        p = (pe, i) if d == 0 else (i, pe)
                        bs[d, e, i] = 2 if coded(m, *q) or coded(o, *p) else (1 if differs(o, p, m, q) else 0)

            def edge(planeno, d, e, chroma, comp_off):
                o = nb[d] if e == 0 else m
                if chroma:
                    qpav = (cqp(int(o["qp"]), comp_off) + cqp(int(m["qp"]), comp_off) + 1) >> 1
                else:
                    qpav = (int(o["qp"]) + int(m["qp"]) + 1) >> 1
                ia = min(max(qpav + int(sp["alpha_offset"]), 0), 51)
                ib = min(max(qpav + int(sp["beta_offset"]), 0), 51)
                alpha, beta = A[ia] << (bd - 8), Bt[ib] << (bd - 8)
                if alpha == 0 or beta == 0:
                    return
                a = pl[planeno]
                n = 8 if chroma else 16
                x0, y0 = (mbx * 8, mby * 8) if chroma else (mbx * 16, mby * 16)
                pos = 2 * e if chroma else 4 * e  # edge position inside the macroblock
                for ln in range(n):
                    b = int(bs[d, e, ln // (n // 4)])
                    if b == 0:
                        continue
                    tc0 = (max(T[ia][b], 0) << (bd - 8)) if b < 4 else 0
                    offs = range(-4, 4)
                    coords = []
                    for k in offs:
                        if chroma and (k < -2 or k > 1):
                            coords.append(None)
                        elif d == 0:
                            coords.append((y0 + ln, x0 + pos + k))
                        else:
                            coords.append((y0 + pos + k, x0 + ln))
                    filter_line(a, coords, b, tc0, alpha, beta, chroma, bool(o["keep"]), bool(m["keep"]))

            for d in (0, 1):
                for e in range(4):
                    if (e == 0 and not ok[d]) or (m["t8x8"] and e % 2 == 1) or not bs[d, e].any():
                        continue
                    edge(0, d, e, False, 0)
            for comp in (0, 1):
                for d in (0, 1):
                    for e in (0, 2):
                        if (e == 0 and not ok[d]) or not bs[d, e].any():
                            continue
                        edge(1 + comp, d, e, True, int(sp["chroma_qp_offset"][comp]))
    dt = y.dtype
    return pl[0].astype(dt), pl[1].astype(dt), pl[2].astype(dt)


# ---- CPU: the oracle ---------------------------------------------------------------------------------

def test_oracle_tables_equal_the_reference_fixture(oracle_lib):
    a, b, t, c = (np.zeros(n, dtype=np.uint8) for n in (52, 52, 156, 22))
    oracle_lib.oracle_dbk_tables(a.ctypes.data, b.ctypes.data, t.ctypes.data, c.ctypes.data)
    assert a.tolist() == TABLES["alpha"] and b.tolist() == TABLES["beta"] and c.tolist() == TABLES["chroma_qp"]
    assert t.reshape(52, 3).tolist() == [[max(v, 0) for v in row[1:]] for row in TABLES["tc0"]]


@pytest.mark.parametrize("mb_w,mb_h,nslices,bd,seed", [(3, 2, 2, 8, 1), (2, 3, 3, 8, 2), (4, 3, 2, 10, 3),
                                                       (3, 3, 1, 8, 4), (2, 2, 4, 10, 5)])
def test_oracle_matches_python_statement(oracle_lib, mb_w, mb_h, nslices, bd, seed):
    rng = np.random.default_rng(seed)
    y, cb, cr = planes(rng, mb_w, mb_h, bd)
    mbs, slices = records(rng, mb_w, mb_h, nslices, bd)
    st = InterStage(mb_w * 16, mb_h * 16, lib=oracle_lib, bd=bd)
    got = st.deblock(y, cb, cr, mbs, slices)
    want = py_deblock(y, cb, cr, mbs, slices, mb_w, mb_h, bd)
    for g, w, name in zip(got, want, ("Y", "Cb", "Cr")):
        assert np.array_equal(g, w), f"{name} differs at {np.argwhere(g != w)[:4].tolist()}"
    assert any(not np.array_equal(g, x) for g, x in zip(got, (y, cb, cr)))  # the case filtered something


def test_oracle_encoder_slices_filter_and_low_qp_leaves_alone(oracle_lib):
    rng = np.random.default_rng(9)
    y, cb, cr = planes(rng, 3, 2)
    mbs, _ = records(rng, 3, 2, 1, slice_rows=True)
    st = InterStage(48, 32, lib=oracle_lib)
    got = st.deblock(y, cb, cr, mbs, encoder_slices(1))
    assert np.array_equal(got[0], py_deblock(y, cb, cr, mbs, encoder_slices(1), 3, 2, 8)[0])
    mbs["qp"] = 10  # indexA below 16: alpha' = 0, nothing is filtered
    got = st.deblock(y, cb, cr, mbs, encoder_slices(1))
    assert all(np.array_equal(g, x) for g, x in zip(got, (y, cb, cr)))


def test_oracle_rejects_a_slice_id_beyond_the_table(oracle_lib):
    rng = np.random.default_rng(3)
    y, cb, cr = planes(rng, 2, 2)
    mbs, slices = records(rng, 2, 2, 2)
    mbs["slice"][3] = 3
    st = InterStage(32, 32, lib=oracle_lib)
    with pytest.raises(IronavError) as e:
        st.deblock(y, cb, cr, mbs, slices)
    assert e.value.status == 2


# ---- GPU: the kernel against the oracle ------------------------------------------------------------------

def _both(oracle_lib, cuda_lib, mb_w, mb_h, nslices, bd, seed, slice_rows=False, enc=False):
    rng = np.random.default_rng(seed)
    y, cb, cr = planes(rng, mb_w, mb_h, bd)
    mbs, slices = records(rng, mb_w, mb_h, nslices, bd, slice_rows=slice_rows)
    if enc:
        slices = encoder_slices(nslices)
    o = InterStage(mb_w * 16, mb_h * 16, lib=oracle_lib, bd=bd)
    c = InterStage(mb_w * 16, mb_h * 16, lib=cuda_lib, bd=bd)
    return o.deblock(y, cb, cr, mbs, slices), c.deblock(y, cb, cr, mbs, slices), (y, cb, cr)


@pytest.mark.gpu
@pytest.mark.parametrize("mb_w,mb_h,nslices,bd,seed,rows,enc", [
    (1, 1, 1, 8, 11, False, False), (2, 1, 2, 8, 12, False, False), (1, 3, 2, 10, 13, False, False),
    (22, 18, 2, 8, 14, True, True), (22, 18, 5, 8, 15, False, False), (22, 18, 3, 10, 16, False, False),
    (120, 68, 8, 8, 17, True, True), (120, 68, 8, 10, 18, True, False), (80, 45, 40, 8, 19, False, False),
])
def test_gpu_deblock_matches_oracle(oracle_lib, cuda_lib, mb_w, mb_h, nslices, bd, seed, rows, enc):
    want, got, src = _both(oracle_lib, cuda_lib, mb_w, mb_h, nslices, bd, seed, rows, enc)
    for g, w, name in zip(got, want, ("Y", "Cb", "Cr")):
        assert np.array_equal(g, w), f"{name} differs at {np.argwhere(g != w)[:4].tolist()}"
    if mb_w * mb_h >= 20:  # (tiny random cases may leave every edge alone)
        assert any(not np.array_equal(w, x) for w, x in zip(want, src))


@pytest.mark.gpu
def test_gpu_deblock_device_form(oracle_lib, cuda_lib):
    import torch

    rng = np.random.default_rng(21)
    mb_w, mb_h = 40, 23
    y, cb, cr = planes(rng, mb_w, mb_h, 10)
    mbs, slices = records(rng, mb_w, mb_h, 3, 10, slice_rows=True)
    want = InterStage(mb_w * 16, mb_h * 16, lib=oracle_lib, bd=10).deblock(y, cb, cr, mbs, slices)
    c = InterStage(mb_w * 16, mb_h * 16, lib=cuda_lib, bd=10)
    c.set_stream(torch.cuda.current_stream().cuda_stream)
    # the planes inside larger buffers: strides beyond the picture width
    ty = torch.zeros((mb_h * 16, mb_w * 16 + 32), dtype=torch.int16, device="cuda")
    tc = torch.zeros((2, mb_h * 8, mb_w * 8 + 16), dtype=torch.int16, device="cuda")
    ty[:, : mb_w * 16] = torch.from_numpy(y.view(np.int16)).cuda()
    tc[0, :, : mb_w * 8] = torch.from_numpy(cb.view(np.int16)).cuda()
    tc[1, :, : mb_w * 8] = torch.from_numpy(cr.view(np.int16)).cuda()
    tm = torch.from_numpy(mbs.view(np.uint8)).cuda()
    c.deblock_device(ty.data_ptr(), ty.shape[1], tc[0].data_ptr(), tc[1].data_ptr(), tc.shape[2], tm.data_ptr(), slices)
    c.sync()
    got = (ty[:, : mb_w * 16].cpu().numpy().view(np.uint16), tc[0, :, : mb_w * 8].cpu().numpy().view(np.uint16),
           tc[1, :, : mb_w * 8].cpu().numpy().view(np.uint16))
    for g, w in zip(got, want):
        assert np.array_equal(g, w)


@pytest.mark.gpu
def test_gpu_deblock_rejects_a_slice_id_beyond_the_table(cuda_lib):
    rng = np.random.default_rng(3)
    y, cb, cr = planes(rng, 4, 3)
    mbs, slices = records(rng, 4, 3, 2)
    mbs["slice"][5] = 7
    c = InterStage(64, 48, lib=cuda_lib)
    with pytest.raises(IronavError) as e:
        c.deblock(y, cb, cr, mbs, slices)
    assert e.value.status == 2
    mbs["slice"][5] = 1
    c.deblock(y, cb, cr, mbs, slices)  # the context is usable after the error


@pytest.mark.gpu
def test_gpu_deblock_device_form_checks_alignment(cuda_lib):
    import torch

    c = InterStage(64, 48, lib=cuda_lib)
    y = torch.zeros((48, 80), dtype=torch.uint8, device="cuda")
    ch = torch.zeros((2, 24, 40), dtype=torch.uint8, device="cuda")
    m = torch.zeros(c.nmb * 192, dtype=torch.uint8, device="cuda")
    from ironav_b200.synth import dbk_encoder_slices

    s = dbk_encoder_slices(1)
    c.deblock_device(y.data_ptr(), 80, ch[0].data_ptr(), ch[1].data_ptr(), 40, m.data_ptr(), s)  # aligned: accepted
    c.sync()
    for args in [(y.data_ptr(), 72, ch[0].data_ptr(), ch[1].data_ptr(), 40),      # luma rows 72 bytes apart
                 (y.data_ptr() + 4, 80, ch[0].data_ptr(), ch[1].data_ptr(), 40),  # luma base off a 16-byte boundary
                 (y.data_ptr(), 80, ch[0].data_ptr(), ch[1].data_ptr(), 36)]:     # chroma rows 36 samples apart
        with pytest.raises(IronavError) as e:
            c.deblock_device(*args, m.data_ptr(), s)
        assert e.value.status == 3



@pytest.mark.gpu
@pytest.mark.parametrize("bd", [8, 10])
def test_gpu_batched_deblock_matches_single_streams(oracle_lib, cuda_lib, bd):
    """Four streams of different sizes and slice layouts (encoder bands, a slice per row, slice ids drawn per
    macroblock with disabled and edge-only filtering) deblocked by one batched call: each stream's planes are
    those of its own call (and the first stream's the oracle's); twice, the progress words cleared each time."""
    import torch

    from ironav_b200.inter import InterBatch, InterStage
    from ironav_b200.synth import dbk_planes, dbk_records

    rng = np.random.default_rng(77 + bd)
    streams = [(352, 288, 2, True), (1920, 1080, 8, True), (176, 144, 9, True), (640, 360, 3, False)]
    stream = torch.cuda.Stream()
    stages, inputs, want = [], [], []
    for (w, h, ns, rows) in streams:
        st = InterStage(w, h, nslices=ns, lib=cuda_lib, bd=bd)
        st.set_stream(stream.cuda_stream)
        planes = dbk_planes(rng, st.mb_w, st.mb_h, bd)
        m, s = dbk_records(rng, st.mb_w, st.mb_h, ns, bd, slice_rows=rows)
        stages.append(st)
        inputs.append((planes, m, s))
        want.append(st.deblock(*planes, m, s))
    o = InterStage(352, 288, nslices=2, lib=oracle_lib, bd=bd)
    planes, m, s = inputs[0]
    for a, b in zip(want[0], o.deblock(*planes, m, s)):
        assert np.array_equal(a, b)
    batch = InterBatch(stages)
    d_m = [torch.from_numpy(m.view(np.uint8)).cuda() for _, m, _ in inputs]
    for _ in range(2):
        d_p = [[torch.from_numpy(a.view(np.int16) if bd == 10 else a.copy()).cuda() for a in planes] for planes, _, _ in inputs]
        torch.cuda.synchronize()
        batch.deblock([p[0].data_ptr() for p in d_p], [p[0].shape[1] for p in d_p], [p[1].data_ptr() for p in d_p],
                      [p[2].data_ptr() for p in d_p], [p[1].shape[1] for p in d_p], [t.data_ptr() for t in d_m],
                      [s for _, _, s in inputs])
        batch.sync()
        for k, (p, w) in enumerate(zip(d_p, want)):
            for name, a, b in zip("Y Cb Cr".split(), p, w):
                got = a.cpu().numpy().view(np.uint16) if bd == 10 else a.cpu().numpy()
                assert np.array_equal(got, b), f"stream {k} {streams[k]}: {name} differs at {np.argwhere(got != b)[:4].tolist()}"
    batch.close()
