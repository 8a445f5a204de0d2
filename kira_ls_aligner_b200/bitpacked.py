"""Host-side 2-bit packing used to build sieve jobs (src/alignment/bitpacked.rs:1-119).

These are the producer side of ``CudaJob`` (what the aligner does on its rayon
pool before dispatch, src/pipeline/stage4_alignment.rs:1280-1304); the scan
itself runs on the GPU.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

_CODE = np.zeros(256, np.uint8)
_VALID = np.zeros(256, bool)
for _c, _v in zip(b"ACGTacgt", (0, 1, 2, 3, 0, 1, 2, 3)):
    _CODE[_c] = _v
    _VALID[_c] = True


@dataclass
class PackedDna:
    """bitpacked.rs:22-33: bits[i] holds bases 4i..4i+3 low-bit first."""
    bits: bytes
    len: int
    valid: bool

    @classmethod
    def pack(cls, seq: bytes) -> "PackedDna":
        a = np.frombuffer(bytes(seq), np.uint8)
        codes = _CODE[a]
        valid = bool(_VALID[a].all())
        n = len(a)
        pad = (-n) % 4
        c = np.concatenate([codes, np.zeros(pad, np.uint8)]).reshape(-1, 4)
        packed = (c[:, 0] | (c[:, 1] << 2) | (c[:, 2] << 4) | (c[:, 3] << 6)).astype(np.uint8)
        return cls(packed.tobytes(), n, valid)

    def pre_shifted_window(self) -> list:
        """bitpacked.rs:47-52 / 95-119: phases at bit offsets 0, 2, 4, 6."""
        b = np.frombuffer(self.bits, np.uint8).astype(np.uint16)
        nxt = np.concatenate([b[1:], np.zeros(1, np.uint16)])
        out = [self.bits]
        for off in (2, 4, 6):
            out.append((((b >> off) | (nxt << (8 - off))) & 0xFF).astype(np.uint8).tobytes())
        return out
