"""Plain-Python decoder of the Q8-stripe layout (test infrastructure).

The layout has no reference counterpart; this restates its decode rule (see
mv_q8_view in include/matvans.h and matvans_b200/csrc/host_q8.cpp) in the most
direct form, so the C++ encoder can be checked on the CPU.  Small sizes only.
"""
import numpy as np


def decode(enc):
    rows, cols = enc["rows"], enc["cols"]
    sq, nseg, local = enc["seg_quads"], enc["nseg"], enc["local"]
    qtot = (cols + 3) // 4
    stripes = (rows + 31) // 32
    blocks, blk_off = enc["blocks"], enc["blk_off"]
    tbl, tbl_off = enc["tbl"].astype(np.uint32), enc["tbl_off"]
    W = np.zeros((stripes * 32, qtot * 4), np.int8)
    for s in range(stripes):
        for g in range(nseg):
            b = s * nseg + g
            o0, o1 = int(blk_off[b]), int(blk_off[b + 1])
            blk = blocks[o0 * 32:o1 * 32].reshape(-1, 32)
            nq = min(sq, qtot - g * sq)
            for l in range(32):
                row = s * 32 + l
                t = row if local else 0
                ents = tbl[tbl_off[t]:tbl_off[t + 1]]
                lut = []
                for e in ents:
                    sym, f = int(e & 0xFF), int(e >> 8)
                    lut += [(sym, f, j) for j in range(f)]
                assert len(lut) == 256
                S = (int(blk[1, l]) << 32) | int(blk[0, l])
                k = 0
                P = None
                for i in range(nq):
                    if S >> 32 == 0:
                        S = (S << 32) | int(blk[2 + k, l])
                        k += 1
                    lo = S & 0xFFFFFFFF
                    ents4 = [lut[(lo >> (8 * j)) & 0xFF] for j in range(4)]
                    f = [e[1] for e in ents4]
                    r = [e[2] for e in ents4]
                    P = f[0] * f[1] * f[2] * f[3]
                    ns = r[0] + f[0] * (r[1] + f[1] * (r[2] + f[2] * r[3]))
                    S = (S >> 32) * P + ns
                    q = g * sq + i
                    for j in range(4):
                        W[row, 4 * q + j] = np.int8(np.uint8(ents4[j][0]).view(np.int8))
                assert S == P, (s, g, l)
                assert k <= blk.shape[0] - 2
    return W[:rows, :cols]
