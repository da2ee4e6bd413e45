"""The learned form of the P-picture analysis (the north star's form 4): the proposer network (ironav_b200.proposer)
proposes, for every macroblock, 4 candidate vectors and its partitioning class, and the analysis judges them by
the exact integer cost (ironav_set_learned): every integer vector within +-2 samples of each proposal is scored by
SAD + lambda * bits, the best is refined by the plain search's sub-sample steps, and the plain search takes over
when the class is not P_Skip or 16x16 or when no proposal does as well as the predictor's own start plus a margin.
The decisions stay those of an exact-cost encoder: the network only chooses where to look.

Training data comes from the plain search itself: the device encoder (decide mode, the plain search) codes seeded
synthetic sequences of the 1080p generator on seeds other than the benchmark's, and each P picture's source, its
reference (the previous filtered reconstruction) and the decisions (vector of the first partition; class P_Skip,
16x16, 16x8, 8x16 or 8x8; intra macroblocks left out) stay on the device as samples. Training is Adam on batches
of macroblocks drawn across all the pictures.

Evaluation codes the benchmark's own sequence with the plain search and with the learned form at the same QP and
compares bytes, luma PSNR, the fallback rate and the analysis rate.
"""
from __future__ import annotations

import time

import numpy as np

from .encoder import DeviceEncoder
from .inter import KIND_INTER
from .proposer import SAMPLE_DTYPE, Proposer, _check
from .synth import CONFIGS, Sequence

TRAIN_SEED = 0x1A2C0000  # training sequences: TRAIN_SEED + k (the benchmark's sequences use 0x1A2B....)
CLASS_NAMES = ("P_Skip", "16x16", "16x8", "8x16", "8x8")


def decision_targets(codes: np.ndarray) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """The training targets of a P picture's decisions (MBCODE_DTYPE): (keep, mv, cls) with keep the inter
    macroblocks (P_Skip included), mv the first partition's vector (quarter samples, int16 [n, 2]) and cls the
    partitioning class (0 P_Skip, 1 16x16, 2 16x8, 3 8x16, 4 8x8)."""
    keep = codes["kind"] == KIND_INTER
    cls = np.where(codes["skip"] != 0, 0, codes["part"].astype(np.int32) + 1).astype(np.uint8)
    mv = codes["mvs"][:, 0, :].astype(np.int16)
    return keep, mv, cls


def picture_samples(d_cur: int, d_ref: int, width: int, height: int, stride: int, ref_stride: int) -> np.ndarray:
    """The samples (SAMPLE_DTYPE) of every macroblock of a picture, in raster order."""
    mb_w, mb_h = (width + 15) // 16, (height + 15) // 16
    s = np.zeros(mb_w * mb_h, dtype=SAMPLE_DTYPE)
    s["cur"], s["ref"] = d_cur, d_ref
    s["w"], s["h"], s["stride"], s["ref_stride"] = width, height, stride, ref_stride
    s["mbx"] = np.tile(np.arange(mb_w, dtype=np.int32), mb_h)
    s["mby"] = np.repeat(np.arange(mb_h, dtype=np.int32), mb_w)
    return s


class TrainingSet:
    """Pictures on the device with their samples and targets (host arrays of the kept macroblocks)."""

    def __init__(self):
        import torch

        self.torch = torch
        self.pictures = []  # (cur tensor, ref tensor): kept alive for the samples' pointers
        self.samples, self.mv, self.cls = [], [], []

    def __len__(self) -> int:
        return sum(len(s) for s in self.samples)

    def collect(self, sequences: int = 3, frames: int = 11, qps=(22, 27, 32), config: str = "1080p", size=None,
                nslices: int = 8, log=None) -> "TrainingSet":
        """Codes `sequences` seeded sequences of `config` at each QP with the plain search and keeps every P
        picture as training data."""
        torch = self.torch
        w0, h0 = CONFIGS[config][:2] if size is None else size
        for k in range(sequences):
            seq = Sequence.config(config, frames, seed=TRAIN_SEED + k, size=size)
            frames_y = [seq.frame(t) for t in range(frames)]
            for qp in qps:
                enc = DeviceEncoder(w0, h0, qp, nslices=min(nslices, (h0 + 15) // 16))
                try:
                    ref = None
                    for t in range(frames):
                        cb, cr = seq.chroma(t)
                        enc.encode(frames_y[t], cb, cr)
                        if t > 0 and ref is not None:
                            codes = enc.codes()
                            keep, mv, cls = decision_targets(codes)
                            cur = torch.from_numpy(frames_y[t]).to(enc.d_rec.device)
                            smp = picture_samples(cur.data_ptr(), ref.data_ptr(), w0, h0, w0, ref.shape[1])
                            self.pictures.append((cur, ref))
                            self.samples.append(smp[keep])
                            self.mv.append(mv[keep])
                            self.cls.append(cls[keep])
                        # the filtered reconstruction is the next picture's reference
                        enc.st.sync()
                        ref = enc.d_rec.clone()
                finally:
                    enc.close()
                if log:
                    log(f"collected seed {k} qp {qp}: {len(self)} samples")
        self._flat = None
        return self

    def flat(self):
        if getattr(self, "_flat", None) is None:
            self._flat = (np.concatenate(self.samples), np.concatenate(self.mv), np.concatenate(self.cls))
        return self._flat

    def class_counts(self) -> np.ndarray:
        return np.bincount(self.flat()[2], minlength=5)


def train(prop: Proposer, data: TrainingSet, samples: int = 2_000_000, batch: int = 512, lr: float = 1e-3,
          lr_head: float | None = None, seed: int = 0x1A2C, log=None, log_every: int = 500) -> list[dict]:
    """Adam on `samples` samples drawn (without replacement within an epoch) from the training set, `batch` a
    step. Returns the losses and the partition accuracy of the first step, then their means over every 50th
    step of each interval of `log_every` steps."""
    torch = prop.torch
    smp, mv, cls = data.flat()
    n_all = len(smp)
    rng = np.random.default_rng(seed)
    order = rng.permutation(n_all)
    pos = 0
    d_mv = torch.zeros((batch, 2), dtype=torch.int16, device=prop.dev)
    d_cls = torch.zeros(batch, dtype=torch.uint8, device=prop.dev)
    hist = []
    acc = np.zeros(3)
    nacc = 0
    steps = max(1, samples // batch)
    t0 = time.perf_counter()
    for step in range(steps):
        if pos + batch > n_all:
            order = rng.permutation(n_all)
            pos = 0
        idx = order[pos:pos + batch]
        pos += batch
        with torch.cuda.stream(prop.stream):
            d_mv.copy_(torch.from_numpy(mv[idx]))
            d_cls.copy_(torch.from_numpy(cls[idx]))
        prop.sums.zero_()
        prop.train_step(smp[idx], d_mv, d_cls, lr=lr, lr_head=lr_head)
        if step == 0 or (step + 1) % 50 == 0 or step + 1 == steps:
            acc += prop.sums.cpu().numpy() / batch
            nacc += 1
        if (step == 0 or (log_every and ((step + 1) % log_every == 0 or step + 1 == steps))) and nacc:
            rec = {"step": step + 1, "samples": (step + 1) * batch, "mv_loss": acc[0] / nacc, "part_loss": acc[1] / nacc,
                   "part_acc": acc[2] / nacc, "seconds": time.perf_counter() - t0}
            hist.append(rec)
            if log:
                log(rec)
            acc[:] = 0
            nacc = 0
    prop.check_errors()
    return hist


class LearnedJudge:
    """The learned form inside a device encoder: before each P picture, the proposer's forward pass over every
    macroblock (cur = the picture, ref = the newest reference, the encoder's filtered reconstruction) and the
    judge's inputs, set on the encoder's context. Counters: judged, class fallbacks, cost fallbacks."""

    def __init__(self, prop: Proposer, enc: DeviceEncoder, margin: int = 0, min_conf: float = 0.0, timed: bool = False):
        torch = prop.torch
        self.prop, self.enc, self.margin, self.min_conf = prop, enc, margin, min_conf
        st = enc.st
        self.n = st.nmb
        dev = prop.dev
        self.cands = torch.zeros((self.n, 8), dtype=torch.int16, device=dev)
        self.cls = torch.zeros(self.n, dtype=torch.uint8, device=dev)
        self.stats = torch.zeros(3, dtype=torch.int32, device=dev)
        self._samples = {}  # device sample arrays by (d_y, stride)
        self.timed = timed
        self.ms = []  # per picture: the proposer's time (ms), when timed
        prop.stream = enc.stream
        st._check(enc.lib.ironav_set_learned(st.ctx, self.cands.data_ptr(), self.cls.data_ptr(), margin, self.stats.data_ptr()),
                  "ironav_set_learned")
        enc.before_p = self

    def _device_samples(self, d_y: int, stride: int):
        key = (d_y, stride)
        if key not in self._samples:
            st = self.enc.st
            smp = picture_samples(d_y, self.enc.d_rec.data_ptr(), st.width, st.height, stride, self.enc.d_rec.shape[1])
            self._samples[key] = self.prop.torch.from_numpy(smp.view(np.uint8)).to(self.prop.dev)
        return self._samples[key]

    def __call__(self, enc: DeviceEncoder, d_y: int, stride: int) -> None:
        torch = self.prop.torch
        d = self._device_samples(d_y, stride)
        if self.timed:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(enc.stream)
        self.prop.set_samples_device(d.data_ptr(), self.n)
        self.prop.forward(self.n)
        self.prop.propose(self.n, self.cands.data_ptr(), self.cls.data_ptr(), self.min_conf)
        if self.timed:
            e1.record(enc.stream)
            e1.synchronize()
            self.ms.append(e0.elapsed_time(e1))

    def counters(self) -> dict:
        s = self.stats.cpu().numpy()
        return {"judged": int(s[0]), "class_fallback": int(s[1]), "cost_fallback": int(s[2])}

    def detach(self) -> None:
        st = self.enc.st
        st._check(self.enc.lib.ironav_set_learned(st.ctx, None, None, 0, None), "ironav_set_learned")
        self.enc.before_p = None


def psnr(a: np.ndarray, b: np.ndarray, peak: float = 255.0) -> float:
    mse = float(np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2))
    return float("inf") if mse == 0 else 10.0 * np.log10(peak * peak / mse)


def encode_sequence(seq: Sequence, qp: int, frames: int, prop: Proposer | None = None, margin: int = 0, min_conf: float = 0.0,
                    nslices: int = 8) -> dict:
    """Codes `frames` pictures of `seq` with the device encoder (plain search, or the learned form with `prop`):
    total bytes, mean luma PSNR, the learned form's counters and proposer time."""
    w, h = seq.width, seq.height
    enc = DeviceEncoder(w, h, qp, nslices=nslices)
    judge = LearnedJudge(prop, enc, margin=margin, min_conf=min_conf, timed=True) if prop is not None else None
    total, ps = 0, []
    try:
        for t in range(frames):
            y = seq.frame(t)
            cb, cr = seq.chroma(t)
            total += len(enc.encode(y, cb, cr))
            ry = enc.recon()[0]
            ps.append(psnr(ry[:h, :w], y))
        out = {"qp": qp, "frames": frames, "bytes": total, "psnr_y": float(np.mean(ps))}
        if judge is not None:
            out.update(judge.counters())
            out["proposer_ms_per_picture"] = float(np.mean(judge.ms)) if judge.ms else None
            judge.detach()
        return out
    finally:
        enc.close()


def analysis_rate(prop: Proposer, seq: Sequence, qp: int, frames: int, margin: int = 0, min_conf: float = 0.0, nslices: int = 8,
                  reps: int = 3) -> dict:
    """Auto-mode analysis (ironav_analyse_picture_auto_device) of pictures 1..frames-1 of `seq`, each from the
    previous source picture, with the plain search and with the learned form (the proposer's input, forward
    pass and proposals, then the analysis with the judge), timed by CUDA events on one stream: macroblocks per
    second of each, the proposer's share, and the judge's counters. The reference's planes are built before
    the timed region in both."""
    import torch

    from .inter import MBRESULT_DTYPE, MBSTATE_DTYPE, InterStage

    w, h = seq.width, seq.height
    st = InterStage(w, h, nslices=nslices)
    stream = torch.cuda.Stream()
    st.set_stream(stream.cuda_stream)
    old_stream = prop.stream
    prop.stream = stream
    dev = prop.dev
    try:
        pics = [torch.from_numpy(seq.frame(t)).to(dev) for t in range(frames)]
        n = st.nmb
        d_states = torch.zeros(n * MBSTATE_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        d_out = torch.zeros(n * MBRESULT_DTYPE.itemsize, dtype=torch.uint8, device=dev)
        cands = torch.zeros((n, 8), dtype=torch.int16, device=dev)
        cls = torch.zeros(n, dtype=torch.uint8, device=dev)
        stats = torch.zeros(3, dtype=torch.int32, device=dev)
        samples = {}
        ms = {"plain": 0.0, "learned": 0.0, "proposer": 0.0}
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        pictures = 0
        for t in range(1, frames):
            st.clear_references()
            st.push_reference_device(pics[t - 1].data_ptr(), w, w, h, None)
            st.set_source_device(pics[t].data_ptr(), w)
            st.begin_p_picture(qp, 1)
            smp = samples.setdefault(t, torch.from_numpy(picture_samples(pics[t].data_ptr(), pics[t - 1].data_ptr(), w, h, w, w)
                                                          .view(np.uint8)).to(dev))
            for r in range(reps + 1):
                st._check(st.lib.ironav_set_learned(st.ctx, None, None, 0, None), "ironav_set_learned")
                ev[0].record(stream)
                st.analyse_auto_device(d_states.data_ptr(), d_out.data_ptr())
                ev[1].record(stream)
                ev[1].synchronize()
                plain_ms = ev[0].elapsed_time(ev[1])
                st._check(st.lib.ironav_set_learned(st.ctx, cands.data_ptr(), cls.data_ptr(), margin, stats.data_ptr()),
                          "ironav_set_learned")
                ev[0].record(stream)
                prop.set_samples_device(smp.data_ptr(), n)
                prop.forward(n)
                prop.propose(n, cands.data_ptr(), cls.data_ptr(), min_conf)
                ev[1].record(stream)
                st.analyse_auto_device(d_states.data_ptr(), d_out.data_ptr())
                ev[2].record(stream)
                ev[2].synchronize()
                if r > 0:  # the first round warms up
                    ms["plain"] += plain_ms
                    ms["proposer"] += ev[0].elapsed_time(ev[1])
                    ms["learned"] += ev[0].elapsed_time(ev[2])
                    pictures += 1
        st._check(st.lib.ironav_set_learned(st.ctx, None, None, 0, None), "ironav_set_learned")
        prop.check_errors()
        mbs = n * pictures
        s = stats.cpu().numpy()
        return {"qp": qp, "pictures": pictures, "plain_mb_per_s": mbs / (ms["plain"] * 1e-3),
                "learned_mb_per_s": mbs / (ms["learned"] * 1e-3), "proposer_ms_per_picture": ms["proposer"] / pictures,
                "plain_ms_per_picture": ms["plain"] / pictures, "learned_ms_per_picture": ms["learned"] / pictures,
                "judged": int(s[0]), "class_fallback": int(s[1]), "cost_fallback": int(s[2])}
    finally:
        prop.stream = old_stream
        st.close()


def conv_tflops(prop: Proposer, n: int, reps: int = 5) -> dict:
    """The tensor-core convolutions' rate on a forward pass over n samples (after set_samples): each layer's
    time by CUDA events on the proposer's stream and its algorithmic FLOPs (2 * 2500 * 9 * 32 * cin per sample;
    the padded 50 x 50 raster is what the kernel computes)."""
    torch = prop.torch
    lib, e = prop.lib, prop.err.data_ptr()
    res = {}
    for l, cin in ((1, 16), (2, 32)):
        x = prop.x0 if l == 1 else prop.z[1]
        w, y = prop.wf[l], prop.z[l]
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        for r in range(reps + 2):
            if r == 2:
                ev[0].record(prop.stream)
            _check(lib.ironav_prop_conv3x3(x.data_ptr(), cin, n, w.data_ptr(), prop.views[f"b{l}"].data_ptr(), 1, None, y.data_ptr(), e,
                                           prop._s), "conv")
        ev[1].record(prop.stream)
        ev[1].synchronize()
        ms = ev[0].elapsed_time(ev[1]) / reps
        flops = 2.0 * 2500 * 9 * 32 * cin * n
        res[f"conv_cin{cin}"] = {"ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}
    prop.check_errors()
    return res


def time_proposer(n: int, reps: int = 5) -> dict:
    """The proposer's forward pass, untrained (seeded random weights), on the first n macroblocks of the 1080p
    sequence's second picture against its first: CUDA-event times of the input, the four layers, the head and
    the whole pass, per call."""
    import torch

    seq = Sequence.config("1080p", 2)
    f0, f1 = (torch.from_numpy(seq.frame(t)).cuda() for t in range(2))
    prop = Proposer(max_batch=n)
    smp = picture_samples(f1.data_ptr(), f0.data_ptr(), 1920, 1080, 1920, 1920)[:n]
    prop.set_samples(smp)
    for _ in range(2):
        prop.forward(n)
    torch.cuda.synchronize()
    out = conv_tflops(prop, n, reps=reps)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    conv = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    ev[0].record(prop.stream)
    for _ in range(reps):
        prop.set_samples_device(prop.samples_d.data_ptr(), n)
    ev[1].record(prop.stream)
    for r in range(reps):
        prop.forward(n, conv_events=conv[r])
    ev[2].record(prop.stream)
    ev[2].synchronize()
    prop.check_errors()
    out["input_ms"] = ev[0].elapsed_time(ev[1]) / reps
    out["forward_ms"] = ev[1].elapsed_time(ev[2]) / reps
    out["layers_ms"] = sum(a.elapsed_time(b) for a, b in conv) / reps
    out["head_ms"] = out["forward_ms"] - out["layers_ms"]
    out["samples"] = n
    return out


def main(argv=None) -> int:
    import argparse
    import json

    import torch

    ap = argparse.ArgumentParser(description="Train the learned proposer on the plain search's decisions and compare "
                                             "the learned form with the plain search on the 1080p sequence.")
    ap.add_argument("--sequences", type=int, default=3)
    ap.add_argument("--frames", type=int, default=11)
    ap.add_argument("--samples", type=int, default=2_000_000)
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--margin", type=int, default=0)
    ap.add_argument("--min-conf", default="0", help="comma-separated class-probability floors to evaluate")
    ap.add_argument("--eval-frames", type=int, default=11)
    ap.add_argument("--qps", default="22,27,32")
    ap.add_argument("--save", default=None, help="write the trained parameters (.npz)")
    ap.add_argument("--load", default=None, help="start from saved parameters (.npz) and skip training")
    ap.add_argument("--json", default=None, help="write the results as JSON")
    ap.add_argument("--time-proposer", type=int, default=0, metavar="N",
                    help="only time the untrained proposer's forward pass on N macroblocks of a 1080p picture, and exit")
    a = ap.parse_args(argv)
    if a.time_proposer:
        print(json.dumps(time_proposer(a.time_proposer)), flush=True)
        return 0
    qps = tuple(int(q) for q in a.qps.split(","))
    log = lambda m: print(m, flush=True)  # noqa: E731
    out = {}
    prop = Proposer(max_batch=a.batch)
    if a.load:
        d = np.load(a.load)
        prop.load_state_dict({"params": d["params"], "step": int(d["step"])})
    else:
        t0 = time.perf_counter()
        data = TrainingSet().collect(sequences=a.sequences, frames=a.frames, qps=qps, log=log)
        out["collect_s"] = time.perf_counter() - t0
        out["train_samples_available"] = len(data)
        out["train_class_counts"] = data.class_counts().tolist()
        hist = train(prop, data, samples=a.samples, batch=a.batch, lr=a.lr, log=log)
        out["train"] = hist
        del data
        torch.cuda.empty_cache()
        if a.save:
            st = prop.state_dict()
            np.savez(a.save, params=st["params"], step=st["step"])
    seq = Sequence.config("1080p", a.eval_frames)
    confs = [float(c) for c in a.min_conf.split(",")]
    out["eval"] = []
    for qp in qps:
        plain = encode_sequence(seq, qp, a.eval_frames)
        for conf in confs:
            lrn = encode_sequence(seq, qp, a.eval_frames, prop=prop, margin=a.margin, min_conf=conf)
            rec = {"qp": qp, "min_conf": conf, "plain": plain, "learned": lrn,
                   "bytes_delta_pct": 100.0 * (lrn["bytes"] - plain["bytes"]) / plain["bytes"],
                   "psnr_delta_db": lrn["psnr_y"] - plain["psnr_y"]}
            searched = lrn["judged"] + lrn["class_fallback"] + lrn["cost_fallback"]
            rec["fallback_rate"] = (lrn["class_fallback"] + lrn["cost_fallback"]) / max(1, searched)
            log(rec)
            out["eval"].append(rec)
    out["analysis"] = []
    for qp in qps:
        for conf in confs:
            rec = analysis_rate(prop, seq, qp, a.eval_frames, margin=a.margin, min_conf=conf)
            rec["min_conf"] = conf
            log(rec)
            out["analysis"].append(rec)
    n = (1920 // 16) * (1088 // 16)
    prop._alloc(n)
    out["conv_rate"] = conv_tflops(prop, n)
    log(out["conv_rate"])
    if a.json:
        with open(a.json, "w") as f:
            json.dump(out, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
