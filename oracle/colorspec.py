"""CPU restatement of the DNG colour specification (test infrastructure: only
tests/ use it): DNGColorSpec (PefFile/DNGColorSpec.cs:31-647), the xy ->
temperature conversion of DNGTemperature (PefFile/DNGTemperature.cs:181-258)
and DNGxyCoord (PefFile/DNGxyCoord.cs:79-115), in Python floats (IEEE double)
with the reference's operation order, plus the PEF colour spec of
PEFFile.SetMembers (PefFile/PEFFile.cs:310-312).

Parity is unpinned: the reference's C# cannot run here and its tests hold
no colour vectors; the restatement is checked against libisa.so's host
implementation bit for bit and against properties (white maps to white,
daylight temperatures, interpolation endpoints).
"""
from __future__ import annotations

import math

import numpy as np

# Robertson's isotemperature lines (published table): mired, u, v, slope
ROBERTSON = [
    (0, 0.18006, 0.26352, -0.24341), (10, 0.18066, 0.26589, -0.25479), (20, 0.18133, 0.26846, -0.26876),
    (30, 0.18208, 0.27119, -0.28539), (40, 0.18293, 0.27407, -0.30470), (50, 0.18388, 0.27709, -0.32675),
    (60, 0.18494, 0.28021, -0.35156), (70, 0.18611, 0.28342, -0.37915), (80, 0.18740, 0.28668, -0.40955),
    (90, 0.18880, 0.28997, -0.44278), (100, 0.19032, 0.29326, -0.47888), (125, 0.19462, 0.30141, -0.58204),
    (150, 0.19962, 0.30921, -0.70471), (175, 0.20525, 0.31647, -0.84901), (200, 0.21142, 0.32312, -1.0182),
    (225, 0.21807, 0.32909, -1.2168), (250, 0.22511, 0.33439, -1.4512), (275, 0.23247, 0.33904, -1.7298),
    (300, 0.24010, 0.34308, -2.0637), (325, 0.24702, 0.34655, -2.4681), (350, 0.25591, 0.34951, -2.9641),
    (375, 0.26400, 0.35200, -3.5814), (400, 0.27218, 0.35407, -4.3633), (425, 0.28039, 0.35577, -5.3762),
    (450, 0.28863, 0.35714, -6.7262), (475, 0.29685, 0.35823, -8.5955), (500, 0.30505, 0.35907, -11.324),
    (525, 0.31320, 0.35968, -15.628), (550, 0.32129, 0.36011, -23.325), (575, 0.32931, 0.36038, -40.770),
    (600, 0.33724, 0.36051, -116.45)]

D50 = (0.3457, 0.3585)

ILLUMINANT_T = {1: 5500.0, 2: (3800.0 + 4500.0) * 0.5, 3: 2850.0, 4: 5500.0, 9: 5500.0, 10: 6500.0, 11: 7500.0,
                12: (5700.0 + 7100.0) * 0.5, 13: (4600.0 + 5500.0) * 0.5, 14: (3800.0 + 4500.0) * 0.5,
                15: (3250.0 + 3800.0) * 0.5, 16: (2600.0 + 3250.0) * 0.5, 17: 2850.0, 18: 5500.0, 19: 6500.0,
                20: 5500.0, 21: 6500.0, 22: 7500.0, 23: 5000.0, 24: 3200.0}


def xy_to_xyz(c):
    x = max(0.000001, min(c[0], 0.999999))
    y = max(0.000001, min(c[1], 0.999999))
    if x + y > 0.999999:
        s = 0.999999 / (x + y)
        x *= s
        y *= s
    return [x / y, 1.0, (1.0 - x - y) / y]


def xyz_to_xy(c):
    total = c[0] + c[1] + c[2]
    if total > 0.0:
        return (c[0] / total, c[1] / total)
    return D50


def mul(a, b):
    r = [[0.0] * 3 for _ in range(3)]
    for j in range(3):
        for k in range(3):
            s = 0.0
            for m in range(3):
                s += a[j][m] * b[m][k]
            r[j][k] = s
    return r


def mat_vec(m, v):
    out = []
    for j in range(3):
        s = 0.0
        for k in range(3):
            s += m[j][k] * v[k]
        out.append(s)
    return out


def inv3(m):
    (a00, a01, a02), (a10, a11, a12), (a20, a21, a22) = m
    t = [[a11 * a22 - a21 * a12, a21 * a02 - a01 * a22, a01 * a12 - a11 * a02],
         [a20 * a12 - a10 * a22, a00 * a22 - a20 * a02, a10 * a02 - a00 * a12],
         [a10 * a21 - a20 * a11, a20 * a01 - a00 * a21, a00 * a11 - a10 * a01]]
    det = a00 * t[0][0] + a01 * t[1][0] + a02 * t[2][0]
    if not abs(det) >= 1e-10:
        raise ValueError("singular")
    return [[t[j][k] / det for k in range(3)] for j in range(3)]


def diag(v):
    return [[v[0], 0.0, 0.0], [0.0, v[1], 0.0], [0.0, 0.0, v[2]]]


IDENT = diag([1.0, 1.0, 1.0])


def scaled(s, m):
    return [[m[j][k] * s for k in range(3)] for j in range(3)]


def add(a, b):
    return [[a[j][k] + b[j][k] for k in range(3)] for j in range(3)]


def temperature_of(c):
    u = 2.0 * c[0] / (1.5 - c[0] + 6.0 * c[1])
    v = 3.0 * c[1] / (1.5 - c[0] + 6.0 * c[1])
    last_dt = 0.0
    for index in range(1, 31):
        du, dv = 1.0, ROBERTSON[index][3]
        ln = math.sqrt(1.0 + dv * dv)
        du /= ln
        dv /= ln
        uu = u - ROBERTSON[index][1]
        vv = v - ROBERTSON[index][2]
        dt = -uu * dv + vv * du
        if dt <= 0.0 or index == 30:
            if dt > 0.0:
                dt = 0.0
            dt = -dt
            f = 0.0 if index == 1 else dt / (last_dt + dt)
            return 1.0E6 / (ROBERTSON[index - 1][0] * f + ROBERTSON[index][0] * (1.0 - f))
        last_dt = dt
    return 0.0


def map_white(w1, w2):
    Mb = [[0.8951, 0.2664, -0.1614], [-0.7502, 1.7135, 0.0367], [0.0389, -0.0685, 1.0296]]
    a = [max(x, 0.0) for x in mat_vec(Mb, xy_to_xyz(w1))]
    b = [max(x, 0.0) for x in mat_vec(Mb, xy_to_xyz(w2))]
    A = [[0.0] * 3 for _ in range(3)]
    for j in range(3):
        A[j][j] = max(0.1, min(b[j] / a[j] if a[j] > 0.0 else 10.0, 10.0))
    return mul(mul(inv3(Mb), A), Mb)


def normalize_forward(m):
    xyz = mat_vec(m, [1.0, 1.0, 1.0])
    return mul(mul(diag(xy_to_xyz(D50)), inv3(diag(xyz))), m)


class Spec:
    pass


def find_xyz_to_camera(s, white, want=False):
    T = temperature_of(white)
    if T <= s.t1:
        g = 1.0
    elif T >= s.t2:
        g = 0.0
    else:
        invT = 1.0 / T
        g = (invT - (1.0 / s.t2)) / ((1.0 / s.t1) - (1.0 / s.t2))

    def mix(a, b):
        return a if g >= 1.0 else (b if g <= 0.0 else add(scaled(g, a), scaled(1.0 - g, b)))

    cm = mix(s.cm1, s.cm2)
    if not want:
        return cm
    if s.fm1 is not None and s.fm2 is not None:
        fm = mix(s.fm1, s.fm2)
    else:
        fm = s.fm1 if s.fm1 is not None else s.fm2
    return cm, fm, mix(s.cc1, s.cc2)


def neutral_to_xy(s, neutral):
    last = D50
    for p in range(30):
        cam = find_xyz_to_camera(s, last)
        nxt = xyz_to_xy(mat_vec(inv3(cam), neutral))
        if abs(nxt[0] - last[0]) + abs(nxt[1] - last[1]) < 0.0000001:
            return nxt
        if p == 29:
            nxt = ((last[0] + nxt[0]) * 0.5, (last[1] + nxt[1]) * 0.5)
        last = nxt
    return last


def set_white(s, white):
    cm, fm, cc = find_xyz_to_camera(s, white, want=True)
    cw = mat_vec(cm, xy_to_xyz(white))
    ws = 1.0 / max(cw)
    cw = [max(0.001, min(ws * x, 1.0)) for x in cw]
    p2c = mul(cm, map_white(D50, white))
    scale = max(mat_vec(p2c, xy_to_xyz(D50)))
    p2c = scaled(1.0 / scale, p2c)
    if fm is not None:
        ind = inv3(mul(s.ab, cc))
        rw = mat_vec(ind, cw)
        c2p = mul(mul(fm, inv3(diag(rw))), ind)
    else:
        c2p = inv3(p2c)
    return c2p, cw


def _m(a):
    return None if a is None else [[float(a[j * 3 + k]) for k in range(3)] for j in range(3)]


def dng_color_spec(color_matrix1=None, color_matrix2=None, illuminant1=0, illuminant2=0, forward_matrix1=None,
                   forward_matrix2=None, camera_calibration1=None, camera_calibration2=None, analog_balance=None,
                   as_shot_neutral=None, as_shot_white_xy=None):
    """(camera_to_pcs 3 x 3, camera_white 3, white xy) of DNGColorSpec(tags)."""
    s = Spec()
    s.t1 = ILLUMINANT_T.get(illuminant1, 0.0)
    s.t2 = ILLUMINANT_T.get(illuminant2, 0.0)
    s.cm1 = _m(color_matrix1) or IDENT
    cm2 = _m(color_matrix2)
    s.fm1 = _m(forward_matrix1)
    s.fm2 = _m(forward_matrix2)
    s.cc1 = _m(camera_calibration1) or IDENT
    s.cc2 = _m(camera_calibration2) or IDENT
    s.ab = diag([float(v) for v in analog_balance]) if analog_balance is not None else IDENT
    if s.fm1 is not None:
        s.fm1 = normalize_forward(s.fm1)
    s.cm1 = mul(mul(s.ab, s.cc1), s.cm1)
    if cm2 is None or s.t1 <= 0.0 or s.t2 <= 0.0 or s.t1 == s.t2:
        s.t1 = s.t2 = 5000.0
        s.cm2, s.fm2, s.cc2 = s.cm1, s.fm1, s.cc1
    else:
        if s.fm2 is not None:
            s.fm2 = normalize_forward(s.fm2)
        s.cm2 = mul(mul(s.ab, s.cc2), cm2)
        if s.t1 > s.t2:
            s.t1, s.t2 = s.t2, s.t1
            s.cm1, s.cm2 = s.cm2, s.cm1
            s.fm1, s.fm2 = s.fm2, s.fm1
            s.cc1, s.cc2 = s.cc2, s.cc1
    if as_shot_white_xy is not None:
        white = (float(as_shot_white_xy[0]), float(as_shot_white_xy[1]))
    else:
        vec = [float(v) for v in as_shot_neutral]
        u = 1.0 / max(vec)
        white = neutral_to_xy(s, [u * v for v in vec])
    c2p, cw = set_white(s, white)
    return np.array(c2p), np.array(cw), np.array(white)


def pef_color_spec(white_balance):
    """DNGColorSpec(identity, identity, D50, D50, whiteBalance) of PEFFile.SetMembers."""
    s = Spec()
    s.t1 = s.t2 = 5000.0
    s.cm1 = s.cm2 = IDENT
    s.fm1 = s.fm2 = None
    s.cc1 = s.cc2 = IDENT
    s.ab = IDENT
    vec = [float(np.float32(1.0) / np.float32(w)) for w in white_balance]
    u = 1.0 / max(vec)
    white = neutral_to_xy(s, [u * v for v in vec])
    c2p, cw = set_white(s, white)
    return np.array(c2p), np.array(cw), np.array(white)
