"""CPU check of the plane-staged slow kernel's addressing (k_slow_xt,
oraclev8_b200/csrc/slowx.cuh) and of its launch sizing (slow_xt_seg in
csrc/api.cu), restated here line for line, for every grid the tests and
workloads run it on:

* the y-halo'd row block of a CTA is one or two runs that cover exactly rows
  j0-3 .. j0+R+2 (mod ny);
* w's runs, copied as 16-byte aligned ranges, start on 16 bytes, stay inside
  the w array, and the second piece of a wrapped run lands, aligned, right
  after the first inside the slot's w region;
* the seven-slot ring: every plane a step reads is the one its slot holds,
  a slot is refilled only after the step that read its plane last, and every
  plane issued is waited for before the kernel ends (no copy in flight at
  exit);
* the x-segments cover [0, nx) exactly, each a multiple of 7 but the last.

No GPU is needed; a mistake here would be an out-of-bounds bulk copy on the
device, so the kernel's formulas are checked before any launch.
"""
import pytest

NSM = 148


def seg_of(nx, ny, r, nsm=NSM):
    """slow_xt_seg (csrc/api.cu)."""
    nrow = ny // r
    nseg = max(1, (8 * nsm + nrow - 1) // nrow)
    seg = (nx + nseg - 1) // nseg
    seg = max(21, (seg + 6) // 7 * 7)
    return min(seg, (nx + 6) // 7 * 7)


def row_runs(j0, r, ny):
    """ga, na, nb of k_slow_xt."""
    rh = r + 6
    ga, na, nb = j0 - 3, rh, 0
    if ga < 0:
        na = -ga
        ga += ny
        nb = rh - na
    elif ga + rh > ny:
        na = ny - ga
        nb = rh - na
    return ga, na, nb


def w_runs(px, ny, nz, ga, nb, r):
    """WRun of k_slow_xt: [wa, we) and, wrapped, [w2, w2e) in floats."""
    nw = nz + 1
    rh = r + 6
    cb = px * ny
    w0 = (cb + ga) * nw
    w2 = cb * nw
    wa = w0 & ~3
    we = (cb + ny) * nw if nb else (w0 + rh * nw + 3) & ~3
    w2e = (w2 + nb * nw + 3) & ~3
    return w0, wa, we, w2, w2e


def check_grid(nx, ny, nz, r):
    assert nz in (32, 48, 64, 80) and ny % r == 0 and ny >= r + 6 and nx >= 7
    assert nx * ny * (nz + 1) < 2 ** 31  # the kernel's 32-bit element offsets
    nw, rh = nz + 1, r + 6
    ws = (rh * nw + 8 + 3) // 4 * 4  # the slot's w region (floats)
    total_w = nx * ny * nw
    for j0 in range(0, ny, r):
        ga, na, nb = row_runs(j0, r, ny)
        rows = [ga + i for i in range(na)] + list(range(nb))
        assert rows == [(j0 - 3 + i) % ny for i in range(rh)]
        for px in range(nx):
            w0, wa, we, w2, w2e = w_runs(px, ny, nz, ga, nb, r)
            lead = w0 & 3
            assert lead == (ga * nw) & 3  # the kernel takes one lead for every plane
            assert wa % 4 == 0 and wa >= 0 and we <= total_w and (we - wa) % 4 == 0
            if nb:
                assert we == w0 + na * nw and we % 4 == 0 and w2 % 4 == 0
                assert w2e <= total_w and (w2e - w2) % 4 == 0
                dst2 = we - wa  # where piece 2 lands in the slot (floats)
                assert dst2 == lead + na * nw and dst2 % 4 == 0
                assert dst2 + (w2e - w2) <= ws
            else:
                assert we - wa <= ws
    seg = seg_of(nx, ny, r)
    starts = list(range(0, nx, seg))
    lens = [min(seg, nx - i0) for i0 in starts]
    assert sum(lens) == nx and all(n % 7 == 0 for n in lens[:-1]) and seg % 7 == 0
    for ln in lens:
        check_ring(ln)


def check_ring(ln):
    """The schedule of one segment of length ln: prologue planes 0..6, then
    7 and 8, then plane st + 9 at step st into the slot of plane st + 2."""
    qmax = ln + 5
    slot, issued, waited = [None] * 7, [], set()

    def issue(q, s):
        assert q % 7 == s
        slot[s] = q
        issued.append(q)

    for q in range(min(6, qmax) + 1):
        issue(q, q)
    waited |= set(range(6))
    for q in range(6):
        assert slot[q] == q  # window fill
    released = {0, 1, 2}
    for q in (7, 8):
        if q <= qmax:
            assert q - 7 in released
            issue(q, q - 7)
    for st in range(ln):
        uu = st % 7
        gp = (st // 7) % 2  # the kernel's group parity
        # phase parities of the waits: plane q is the (q // 7)-th fill of its slot
        assert (gp + (uu >= 1)) % 2 == ((st + 6) // 7) % 2
        assert (gp + (uu >= 5)) % 2 == ((st + 2) // 7) % 2
        assert slot[(uu + 6) % 7] == st + 6
        waited.add(st + 6)
        if st + 9 <= qmax:
            assert st + 2 in released  # read for the last time in step st - 1
            issue(st + 9, (uu + 2) % 7)
        assert slot[(uu + 3) % 7] == st + 3 and slot[(uu + 6) % 7] == st + 6
        released.add(st + 3)
    assert set(issued) <= waited


@pytest.mark.parametrize("nx, ny, nz", [
    (48, 24, 80), (64, 40, 32), (96, 16, 64), (40, 12, 48),   # the GPU tests' shapes
    (1024, 1024, 80), (1024, 256, 80), (512, 512, 64),        # the workloads and the slab
    (96, 96, 32), (128, 128, 48), (192, 192, 64), (256, 256, 32), (384, 384, 64)])  # ensemble
def test_plane_staged_slow_kernel_addressing(nx, ny, nz):
    for r in (4, 8):
        if ny % r == 0 and ny >= r + 6:
            check_grid(nx, ny, nz, r)
