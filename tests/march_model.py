"""CPU model of the tcs_march kernel's addressing (used by tests/test_march_model.py).

Transcribes, formula for formula, the launch planning of ``resolve_march`` (tcs_capi.cpp) and the
indexing of the ``tcs_march`` kernel (tcs_kernels.cuh): TMA box coordinates, ring slots, the
per-step wait/issue schedule and every shared-memory read of every thread.  The ring is filled
with global linear indices (or -1 where the TMA box falls outside the tensor) so each read can be
checked against the grid point the stencil needs.  Any out-of-bounds shared-memory access, wrong
element, unaligned TMA coordinate, reuse of a slot still in use or interior point not written
exactly once raises AssertionError.
"""

from __future__ import annotations

import math


def cdiv(a, b):
    return (a + b - 1) // b


def plan(dim, R, c, block, grid, x0, x_lim, y_lim, z_lim, es, smem_optin=232448, num_sms=148, occ=1,
         segments=0, depth=0):
    """resolve_march: returns None when unsupported, else the launch parameters."""
    cx, cy, cz = c
    vec = 16 // es
    TX = block[0] * cx
    if dim == 2:
        STEP, rows = block[1] * cy, 1
    else:
        STEP, rows = block[2] * cz, block[1] * cy + 2 * R
    W = cdiv(TX + 2 * R + vec - 1, vec) * vec
    while (STEP * W * rows * es) % 128:
        W += vec
    if W > 256 or STEP > 256 or rows > 256:
        return None
    plane = W * rows
    chunk_bytes = STEP * plane * es
    K = 1 + cdiv(2 * R, STEP)
    if depth == 0:
        depth = max(1, min(4, cdiv(16384, chunk_bytes)))
    while True:
        nslot = K + depth
        smem = cdiv(nslot * 8, 128) * 128 + 128 + nslot * chunk_bytes
        if smem <= smem_optin or depth == 1:
            break
        depth -= 1
    if smem > smem_optin:
        return None
    ex = max(0, x_lim - x0)
    ey = y_lim - R
    nxt = max(1, cdiv(ex, TX))
    nyt = 1
    M = ey
    if dim == 3:
        nyt = max(1, cdiv(ey, block[1] * cy))
        M = z_lim - R
    nseg = segments
    if nseg == 0:
        nseg = max(1, (num_sms * occ) // max(1, nxt * nyt))
    nseg = min(nseg, max(1, cdiv(M, STEP)))
    seg = cdiv(max(M, 1), nseg)
    seg = cdiv(seg, STEP) * STEP
    nseg = max(1, cdiv(max(M, 1), seg))
    gridb = (nxt, nseg, 1) if dim == 2 else (nxt, nyt, nseg)
    return dict(W=W, STEP=STEP, rows=rows, plane=plane, K=K, nslot=nslot, smem=smem, seg=seg, grid=gridb,
                depth=depth, vec=vec)


def footprint(dim, shape, R, c):
    """Union footprint offsets of one thread tile (order irrelevant here)."""
    cx, cy, cz = c
    pts = set()
    zs = range(-R, R + cz) if dim == 3 else [0]
    for gz in zs:
        for gy in range(-R, R + cy):
            for gx in range(-R, R + cx):
                for ez in range(cz if dim == 3 else 1):
                    for ey in range(cy):
                        for ex in range(cx):
                            rx, ry, rz = gx - ex, gy - ey, gz - ez
                            if shape == "Box":
                                ok = abs(rx) <= R and abs(ry) <= R and abs(rz) <= R
                            elif dim == 2:
                                ok = (abs(rx) <= R and ry == 0) or (abs(ry) <= R and rx == 0)
                            else:
                                ok = ((abs(rx) <= R and ry == 0 and rz == 0) or (abs(ry) <= R and rx == 0 and rz == 0)
                                      or (abs(rz) <= R and rx == 0 and ry == 0))
                            if ok:
                                pts.add((gx, gy, gz))
    return sorted(pts)


def simulate(dim, shape, R, c, block, grid, left_offset, right_offset, aligned, es=8, **plan_kw):
    """Run the model over every CTA; returns the number of outputs written (or None if the
    planner rejects the shape)."""
    cx, cy, cz = c if dim == 3 else (c[0], c[1], 1)
    xdim, ydim = grid[0], grid[1]
    zdim = grid[2] if dim == 3 else 1
    ro = right_offset if aligned else 0
    x0 = R + left_offset
    x_lim = xdim - R - ro
    y_lim = ydim - R
    z_lim = zdim - R if dim == 3 else 1
    p = plan(dim, R, (cx, cy, cz), block, (xdim, ydim, zdim), x0, x_lim, y_lim, z_lim, es, **plan_kw)
    if p is None:
        return None
    W, STEP, plane, K, nslot, seg, vec = p["W"], p["STEP"], p["plane"], p["K"], p["nslot"], p["seg"], p["vec"]
    rows = p["rows"]
    bar_bytes = cdiv(nslot * 8, 128) * 128
    ring_elems = nslot * STEP * plane
    assert bar_bytes + 128 + ring_elems * es == p["smem"]
    # TMA destinations: the ring starts on a 128-byte boundary and every slot is a multiple of 128 B
    assert (STEP * plane * es) % 128 == 0, "TMA destination not 128-byte aligned"
    # the ring, placed after the barriers and rounded up to 128 bytes, ends inside the allocation
    for base in (0, 16, 64):  # possible dynamic shared-memory base offsets (mod 128)
        ring_off = ((base + bar_bytes + 127) // 128) * 128 - base
        assert ring_off + ring_elems * es <= p["smem"]
    chunk_elems = STEP * plane
    ring_planes = nslot * STEP
    TX = block[0] * cx
    fp = footprint(dim, shape, R, (cx, cy, cz))
    written = {}
    gx_, gy_, gz_ = p["grid"]
    for bz in range(gz_):
        for by in range(gy_):
            for bx in range(gx_):
                if dim == 2:
                    mlim, ms, Y0 = y_lim, R + by * seg, 0
                else:
                    TY = block[1] * cy
                    mlim, ms, Y0 = z_lim, R + bz * seg, R + by * TY
                if ms >= mlim:
                    continue
                me = min(ms + seg, mlim)
                nsteps = cdiv(me - ms, STEP)
                nchunks = cdiv(me - ms + 2 * R, STEP)
                X0 = x0 + bx * TX
                xl = (X0 - R) & ~(vec - 1)
                assert xl % vec == 0 and xl >= 0
                ring = [None] * ring_elems
                slot_chunk = [None] * nslot     # which chunk a slot holds
                issued = []

                def issue(j):
                    slot = j % nslot
                    dst = slot * chunk_elems
                    assert 0 <= dst and dst + chunk_elems <= ring_elems
                    slot_chunk[slot] = j
                    issued.append(j)
                    zc = ms - R + j * STEP
                    for q in range(chunk_elems):
                        xx = xl + q % W
                        if dim == 2:
                            yy = zc + q // W
                            gidx = xx + yy * xdim if (xx < xdim and yy < ydim) else -1
                        else:
                            yy = Y0 - R + (q // W) % rows
                            zz = zc + q // plane
                            gidx = (xx + yy * xdim + zz * xdim * ydim
                                    if (xx < xdim and yy < ydim and zz < zdim) else -1)
                        ring[dst + q] = gidx

                for j in range(min(nslot - 1, nchunks)):
                    issue(j)
                ring_base = 0
                for s in range(nsteps):
                    jlo = 0 if s == 0 else s + K - 1
                    jhi = min(s + K - 1, nchunks - 1)
                    for j in range(jlo, jhi + 1):
                        assert j in issued, "wait on a chunk never issued"
                    # chunks needed by this step must be resident
                    for j in range(s, min(s + K, nchunks)):
                        assert slot_chunk[j % nslot] == j, "needed chunk overwritten"
                    j = s + nslot - 1
                    if j < nchunks:
                        assert all(slot_chunk[jj % nslot] == jj for jj in range(s, min(s + K, nchunks)))
                        issue(j)
                        for jj in range(s, min(s + K, nchunks)):
                            assert slot_chunk[jj % nslot] == jj, "issued into a slot still needed"
                    for tz in range(block[2]):
                        for ty in range(block[1]):
                            for tx in range(block[0]):
                                x = X0 + tx * cx
                                col = x - xl
                                if dim == 3:
                                    y = Y0 + ty * cy
                                    row0 = ty * cy + R
                                    lane_ok = x + cx - 1 < x_lim and y + cy - 1 < y_lim
                                    tm = tz * cz
                                else:
                                    lane_ok = x + cx - 1 < x_lim
                                    tm = ty * cy
                                m = ms + s * STEP + tm
                                ok = lane_ok and (m + ((cz if dim == 3 else cy) - 1) < me)
                                if not ok:
                                    continue
                                pb = ring_base + tm
                                if pb >= ring_planes:
                                    pb -= ring_planes
                                for (gx, gy, gz) in fp:
                                    if dim == 2:
                                        rr = pb + (gy + R)
                                        if rr >= ring_planes:
                                            rr -= ring_planes
                                        idx = rr * W + col + gx
                                        want = (x + gx) + (m + gy) * xdim
                                    else:
                                        pp = pb + (gz + R)
                                        if pp >= ring_planes:
                                            pp -= ring_planes
                                        idx = pp * plane + (row0 + gy) * W + col + gx
                                        want = (x + gx) + (y + gy) * xdim + (m + gz) * xdim * ydim
                                    assert 0 <= idx < ring_elems, "shared-memory read out of bounds"
                                    assert ring[idx] == want, "read %r want %r" % (ring[idx], want)
                                for ez in range(cz if dim == 3 else 1):
                                    for ey in range(cy):
                                        for ex in range(cx):
                                            if dim == 2:
                                                o = (x + ex) + (m + ey) * xdim
                                            else:
                                                o = (x + ex) + (y + ey) * xdim + (m + ez) * xdim * ydim
                                            assert 0 <= o < xdim * ydim * zdim
                                            written[o] = written.get(o, 0) + 1
                    ring_base += STEP
                    if ring_base >= ring_planes:
                        ring_base -= ring_planes
    # every interior point written exactly once
    zr = range(R, z_lim) if dim == 3 else [0]
    count = 0
    for z in zr:
        for y in range(R, y_lim):
            for x in range(x0, x_lim):
                o = x + y * xdim + z * xdim * ydim
                assert written.get(o, 0) == 1, "interior point %d written %d times" % (o, written.get(o, 0))
                count += 1
    assert len(written) == count, "a point outside the interior was written"
    return count
