"""Index maps of the two-stage line FFT (csrc/gs_fft.cuh), checked on the host
for every plan the kernels instantiate: the output positions of a line's
threads cover the line once, and the partner Z_{H-k} that the z-forward split
takes by a warp shuffle (csrc/gs_passes.cuh, zfwd_line) is register
R1-1-i of thread P-t, or, for thread 0, register zfwd_partner0(i)."""
import os
import re

from conftest import PKG


def plans():
    src = open(os.path.join(PKG, "csrc", "gs_fft.cuh")).read()
    out = {int(n): (int(a), int(b)) for n, a, b in re.findall(r"GS_PLAN\((\d+),\s*(\d+),\s*(\d+)\)", src)}
    assert out, "no GS_PLAN lines found"
    return out


def out_pos(t, i, r1, r2):
    p = r2  # threads per line
    return (t + p * (i // r2)) + (i % r2) * r1


def partner0(i, r1, r2):
    b, j = divmod(i, r2)
    if b == 0:
        return 0 if j == 0 else r2 - j
    return (r1 // r2 - b) * r2 + (r2 - 1 - j)


def test_output_positions_cover_each_line_once():
    for n, (r1, r2) in plans().items():
        assert r1 * r2 == n and r1 % r2 == 0
        pos = sorted(out_pos(t, i, r1, r2) for t in range(r2) for i in range(r1))
        assert pos == list(range(n)), n


def test_zforward_partner_map():
    for n, (r1, r2) in plans().items():
        p = r2
        for t in range(p):
            for i in range(r1):
                k = out_pos(t, i, r1, r2)
                if k == 0:
                    continue
                tp, ip = (0, partner0(i, r1, r2)) if t == 0 else ((p - t) % p, r1 - 1 - i)
                assert 0 <= ip < r1
                assert out_pos(tp, ip, r1, r2) == (n - k) % n, (n, t, i)
