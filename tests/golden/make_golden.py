"""Generates the golden fixtures under tests/golden/ (run from the repository root:
`python -m tests.golden.make_golden`).

- exp_golomb.json: the code lengths of the values of the reference's exp_golomb_codes_read_back test
  (crates/ironav-codec/src/h264/enc/bitw.rs:110-135), from the definition of ue(v)/se(v) (H.264 9.1):
  ue(v) takes 2*floor(log2(v+1))+1 bits, se(v) codes 2v-1 for v > 0 and -2v otherwise.
- oracle_cif.npz: the oracle's stage outputs on seeded CIF cases (auto-mode decisions and results, and
  replay results on perturbed decisions), with a hash of the inputs. The reference itself has no golden
  MVs, costs or partitions; these fixtures pin the oracle (and, on the GPU, the kernels) against
  regressions.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

UE_VALUES = [0, 1, 2, 3, 7, 254, 255, 65535, 1 << 20]
SE_VALUES = [0, 1, -1, 2, -2, 1000, -1000]

CASES = {
    "cif_qp26": dict(qp=26, refs=[0], src=1, slices=2),
    "cif_qp22_col": dict(qp=22, refs=[1], src=2, slices=2),
    "cif_qp32_fast": dict(qp=32, refs=[0], src=1, slices=2, fast=True),
    "cif_qp20_sub8": dict(qp=20, refs=[1], src=2, slices=1, sub8=True),
    "cif_qp27_3refs": dict(qp=27, refs=[0, 1, 2], src=3, slices=3),
}


def ue_len(v: int) -> int:
    return 2 * (v + 1).bit_length() - 1


def se_len(v: int) -> int:
    return ue_len(2 * v - 1 if v > 0 else -2 * v)


def perturb(states: np.ndarray, nact: int) -> np.ndarray:
    """Decisions a mode decision could have made instead: every 5th macroblock intra, and with
    several references every 3rd inter macroblock on reference 1."""
    s = states.copy()
    s["inter"][::5] = 0
    s["refs"][::5] = -1
    s["mvs"][::5] = 0
    if nact > 1:
        idx = np.arange(len(s))
        sel = (idx % 3 == 1) & (s["inter"] == 1)
        s["refs"][sel] = 1
    return s


def run_case(lib, qp, refs, src, slices, fast=False, sub8=False):
    from ironav_b200.inter import InterStage
    from ironav_b200.synth import Sequence

    seq = Sequence.config("cif", 4)
    frames = {t: seq.frame(t) for t in range(4)}
    h = hashlib.sha256()
    for t in list(refs) + [src]:
        h.update(frames[t].tobytes())

    def decisions_of(t):
        # a reference picture's own decisions (its col vectors): t analysed against t-1 in auto mode
        if t == 0:
            return None
        s1 = InterStage(352, 288, max_refs=1, nslices=slices, lib=lib)
        s1.push_reference(frames[t - 1])
        s1.set_source(frames[t])
        s1.begin_p_picture(qp)
        states, _ = s1.analyse_auto()
        s1.close()
        return states

    st = InterStage(352, 288, max_refs=len(refs), nslices=slices, lib=lib)
    for t in refs:
        st.push_reference(frames[t], col=decisions_of(t))
    st.set_source(frames[src])
    st.begin_p_picture(qp, nrefs_active=len(refs), fast=fast, sub8=sub8)
    states, res = st.analyse_auto()
    rstates = perturb(states, len(refs))
    rres = st.analyse_replay(rstates)
    st.close()
    return h.hexdigest(), states, res, rstates, rres


def main():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from tests.oracle_lib import oracle_library

    ue_bits = [ue_len(v) for v in UE_VALUES]
    se_bits = [se_len(v) for v in SE_VALUES]
    with open(os.path.join(HERE, "exp_golomb.json"), "w") as f:
        json.dump({"ue_values": UE_VALUES, "ue_bits": ue_bits, "se_values": SE_VALUES, "se_bits": se_bits,
                   "total_bits": sum(ue_bits) + sum(se_bits) + 5}, f, indent=1)
    lib = oracle_library()
    out = {}
    for name, case in CASES.items():
        hh, states, res, rstates, rres = run_case(lib, **case)
        out[f"{name}_hash"] = np.array(hh)
        out[f"{name}_states"] = states
        out[f"{name}_results"] = res
        out[f"{name}_rstates"] = rstates
        out[f"{name}_replay"] = rres
    np.savez_compressed(os.path.join(HERE, "oracle_cif.npz"), **out)


if __name__ == "__main__":
    main()
