"""The algorithm of the parallel DNG decoder (imagestackalignator_b200/csrc/raw.cu,
the k_dngf_* kernels) modelled step by step in Python -- byte skipping into
128-byte-aligned regions, 1024-bit chunks decoded from 32 candidate starts,
33-state maps chained in three levels with a reset at each part, the
per-part symbol offsets and the hand-back flag, the differences, the vpred
column sums and the row sums -- and checked against the restated reference
reader (oracle/raw.py, orc_dng_decode) without a GPU. The blocks of the
chaining are made small here (4 chunks, 2 sub-blocks) so that small frames
cross many block and sub-block boundaries; the GPU tests check the kernels
themselves against the same reader."""
import numpy as np
import pytest

import raw as R

STOP = 32
CB = 4    # chunks per block of the composition (1024 on the GPU)
WPB = 2   # sub-blocks per block (32 warps on the GPU)


def parse(part):
    """(data offset, bits, high, wide, clrs, psv, restart, table(list)) of a lossless-JPEG part (minimal, like lj92_start)."""
    part = bytes(bytearray(part))
    pos = 2
    restart = 0x7fffffff
    table = None
    while True:
        tag = part[pos] << 8 | part[pos + 1]
        ln = (part[pos + 2] << 8 | part[pos + 3]) - 2
        d = part[pos + 4:pos + 4 + ln]
        pos += 4 + ln
        if tag == 0xFFC3:
            bits, high, wide, clrs = d[0], d[1] << 8 | d[2], d[3] << 8 | d[4], d[5]
        elif tag == 0xFFC4:
            counts = d[1:17]
            mx = 16
            while mx > 0 and counts[mx - 1] == 0:
                mx -= 1
            t = [0] * (1 + (1 << mx))
            t[0] = mx
            hh = 1
            dp = 17
            for ln_ in range(1, mx + 1):
                for i in range(counts[ln_ - 1]):
                    for j in range(1 << (mx - ln_)):
                        if hh <= 1 << mx:
                            t[hh] = ln_ << 8 | d[dp]
                            hh += 1
                    dp += 1
            table = t
        elif tag == 0xFFDA:
            psv = d[1 + d[0] * 2]
            bits -= d[3 + d[0] * 2] & 15
            break
        elif tag == 0xFFDD:
            restart = d[0] << 8 | d[1]
    return pos, bits, high, wide, clrs, psv, restart, table


def emulate(file, offs, cnts, W, H, tile_w, tile_h, large=True):
    parts = []
    reg = 0
    sbase = 0
    row = col = 0
    for o, c in zip(offs, cnts):
        part = file[o:o + c]
        dpos, bits, high, wide, clrs, psv, restart, table = parse(part)
        n = c - dpos
        parts.append(dict(pos=o + dpos, n=n, reg=reg, sbase=sbase, cs=reg // 128, high=high, jwide=wide * clrs, clrs=clrs, bits=bits,
                          out_row=row, out_col=col, table=table))
        reg += (n + 256 + 127) // 128 * 128
        sbase += high * wide * clrs
        col += tile_w
        if col >= W:
            col = 0
            row += tile_h
    nchunks = reg // 128
    table = parts[0]["table"]
    hmax = table[0]
    adv = [0] * (1 << hmax)
    for i in range(1 << hmax):
        e = table[1 + i]
        clen, cat = e >> 8, e & 255
        if clen:
            adv[i] = clen + (0 if (cat == 16 and large) else cat)
    # 1. unstuff
    us = bytearray(b"\xff" * (nchunks * 128 + 256))
    first = [0] * nchunks
    for P in parts:
        first[P["cs"]] = 1
        src = bytes(bytearray(file[P["pos"]:P["pos"] + P["n"]]))
        o = 0
        for i in range(P["n"]):
            run = 0
            j = i - 1
            while j >= 0 and src[j] == 0xFF:
                run += 1
                j -= 1
            if run % 2 == 0:
                us[P["reg"] + o] = src[i]
                o += 1
    bitsarr = np.unpackbits(np.frombuffer(bytes(us), np.uint8))

    def window(p):  # 32 bits at global bit p
        b = bitsarr[p:p + 32]
        return int("".join(map(str, b)), 2)

    # 2. maps
    nextk = np.zeros((nchunks, 32), np.int64)
    cntk = np.zeros((nchunks, 32), np.int64)
    for i in range(nchunks):
        for k in range(32):
            p = 0 if first[i] else k
            c = 0
            stop = False
            while p < 1024:
                a = adv[window(i * 1024 + p) >> (32 - hmax)]
                if a == 0:
                    stop = True
                    break
                p += a
                c += 1
            nextk[i, k] = STOP if stop else p - 1024
            cntk[i, k] = c
    # 3. compose / chain / walk
    m = np.zeros((nchunks, 33), np.int64)
    m[:, :32] = nextk
    for i in range(nchunks):
        m[i, 32] = m[i, 0] if first[i] else STOP
    nblocks = (nchunks + CB - 1) // CB
    sub = CB // WPB
    sub_map = np.zeros((nblocks, WPB, 33), np.int64)
    block_map = np.zeros((nblocks, 33), np.int64)
    for b in range(nblocks):
        for w in range(WPB):
            for e in range(33):
                s = e
                for q in range(b * CB + w * sub, min(nchunks, b * CB + w * sub + sub)):
                    s = m[q, s]
                sub_map[b, w, e] = s
        for e in range(33):
            s = e
            for w in range(WPB):
                s = sub_map[b, w, s]
            block_map[b, e] = s
    block_in = []
    s = 0
    for b in range(nblocks):
        block_in.append(s)
        s = block_map[b, s]
    sin = np.zeros(nchunks, np.int64)
    loc = np.zeros(nchunks, np.int64)
    btot = []
    for b in range(nblocks):
        s = block_in[b]
        went = []
        for w in range(WPB):
            went.append(s)
            s = sub_map[b, w, s]
        for w in range(WPB):
            s = went[w]
            for q in range(b * CB + w * sub, min(nchunks, b * CB + w * sub + sub)):
                if first[q]:
                    s = 0
                sin[q] = s
                if s == STOP:
                    loc[q] = 0
                    continue
                loc[q] = cntk[q, s]
                s = nextk[q, s]
        seg = loc[b * CB:min(nchunks, b * CB + CB)].copy()
        btot.append(int(seg.sum()))
        loc[b * CB:min(nchunks, b * CB + CB)] = np.cumsum(seg) - seg
    boff = np.concatenate([[0], np.cumsum(btot)])

    def G(i):
        return boff[i // CB] + loc[i] if i < nchunks else boff[nblocks]

    anomaly = False
    g0 = []
    for t, P in enumerate(parts):
        a = P["cs"]
        e = parts[t + 1]["cs"] if t + 1 < len(parts) else nchunks
        g0.append(G(a))
        S = P["high"] * P["jwide"]
        if G(e) - G(a) < S:
            s = sin[e - 1]
            ex = STOP if s == STOP else nextk[e - 1, s]
            if ex != STOP:
                anomaly = True
    diff = np.zeros(sum(P["high"] * P["jwide"] for P in parts) + 8, np.int64)
    cs = [P["cs"] for P in parts]
    for i in range(nchunks):
        p = sin[i]
        if p == STOP:
            continue
        t = max(k for k in range(len(cs)) if cs[k] <= i)
        P = parts[t]
        S = P["high"] * P["jwide"]
        o = G(i) - g0[t]
        while p < 1024 and o < S:
            x = window(i * 1024 + p)
            e = table[1 + (x >> (32 - hmax))]
            clen, cat = e >> 8, e & 255
            if clen == 0:
                break
            if cat == 16 and large:
                d = -32768
                p += clen
            else:
                d = ((x << clen) & 0xFFFFFFFF) >> (32 - cat) if cat else 0
                if cat and ((d >> (cat - 1)) & 1) == 0:
                    d -= (1 << cat) - 1
                p += clen + cat
            diff[P["sbase"] + o] = d & 0xFFFF
            o += 1
    out = np.zeros((H, W), np.uint16)
    err = False
    for P in parts:
        for c in range(P["clrs"]):
            carry = 1 << (P["bits"] - 1)
            for r in range(P["high"]):
                at = P["sbase"] + r * P["jwide"] + c
                carry += diff[at]
                diff[at] = carry & 0xFFFF
        for r in range(P["high"]):
            row = diff[P["sbase"] + r * P["jwide"]: P["sbase"] + (r + 1) * P["jwide"]].copy()
            for c in range(P["clrs"]):
                row[c::P["clrs"]] = np.cumsum(row[c::P["clrs"]]) & 0xFFFF
            if (row >> P["bits"]).any():
                err = True
            orow = P["out_row"] + r
            if orow < H:
                for j in range(P["jwide"]):
                    oc = P["out_col"] + j
                    if oc < W:
                        out[orow, oc] = row[j]
    return anomaly, err, out


def _tiles(img, tw, th, clrs, bits):
    return R.dng_tiles(img, tw, th, clrs=clrs, bits=bits, psv=1)


def _random_entropy(f, offs, cnts, seed, ff, nbytes=None):
    r = np.random.default_rng(seed)
    parts, no, nc, pos = [f[:offs[0]]], [], [], offs[0]
    for o, c in zip(offs, cnts):
        p = f[o:o + c]
        h = parse(p)[0]
        n = nbytes if nbytes is not None else c - h
        d = r.integers(0, 256, n).astype(np.uint8)
        d[r.random(n) < ff] = 0xFF
        q = np.concatenate([p[:h], d])
        no.append(pos); nc.append(len(q)); parts.append(q); pos += len(q)
    return np.concatenate(parts), no, nc


def _check(f, offs, cnts, W, H, tw, th, large=True):
    st, want = R.dng_decode(f, W, H, offs, cnts, tiled=True, tile_w=tw, tile_h=th, large=large)
    anomaly, err, got = emulate(f, offs, cnts, W, H, tw, th, large)
    assert not anomaly
    assert err == (st != 0)
    if st == 0:
        assert np.array_equal(got, want)


@pytest.mark.parametrize("clrs", [1, 2])
def test_model_encoded_tiles(clrs):
    img = np.clip(np.random.default_rng(clrs).normal(3000, 900, (40, 64)), 0, 16383).astype(np.uint16)
    f, offs, cnts = _tiles(img, 32, 20, clrs, 14)
    _check(f, offs, cnts, 64, 40, 32, 20)


@pytest.mark.parametrize("seed", range(6))
def test_model_random_entropy(seed):
    """16-bit frames whose entropy bytes are random: 0xFF runs, empty code entries, early ends."""
    img = np.random.default_rng(9).integers(0, 32768, (40, 64)).astype(np.uint16)
    f, offs, cnts = _tiles(img, 32, 20, 1 + seed % 2, 16)
    f, offs, cnts = _random_entropy(f, offs, cnts, 20 + seed, ff=[0.02, 0.3, 0.6][seed % 3], nbytes=[None, None, 30, None, 5, None][seed])
    _check(f, offs, cnts, 64, 40, 32, 20, large=seed % 2 == 0)
