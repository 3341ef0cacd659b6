"""CPU model of the tcs_pipe kernel's addressing (used by tests/test_kernel_host.py).

Transcribes the planning of ``resolve_pipe`` (tcs_capi.cpp) and the indexing of ``tcs_pipe``
(tcs_kernels.cuh): row width, ring slots and 128-byte TMA destinations, the per-CTA split of the
(tile, plane) work list into pieces, the chunk issue/wait schedule with the CTA's running chunk
counter, and every shared-memory read of every thread.  The ring holds global linear indices (or
-1 outside the tensor) so that each read is checked against the grid point the stencil needs;
every interior output must be written exactly once.
"""

from __future__ import annotations

from march_model import cdiv


def pipe_width(tx, R, lshift, vec, ch, rows, es):
    w = cdiv(tx + 2 * R + lshift, vec) * vec
    while (ch * rows * w * es) % 128:
        w += vec
    return w


def in_plane_points(dim, shape, R, cx, cy):
    """(gx, gy) offsets a thread reads from one plane."""
    ny = cy if dim == 3 else 1
    pts = set()
    if shape == "Box":
        ys = range(-R, R + cy) if dim == 3 else [0]
        for gy in ys:
            for gx in range(-R, R + cx):
                pts.add((gx, gy))
    else:
        for gy in range(ny):
            for gx in range(-R, R + cx):
                pts.add((gx, gy))
        if dim == 3:
            for gx in range(cx):
                for gy in range(-R, R + cy):
                    pts.add((gx, gy))
    return sorted(pts)


def pair_loads(dim, shape, orient, R, cx, cy, lshift):
    """(gx, gy) where tcs_pipe issues a two-element load (load_row in tcs_tile.cuh)."""
    def aligned(gx):
        return cx % 2 == 0 and (lshift + R + gx) % 2 == 0

    segs = []
    if orient == "Column" and dim == 3:
        return []
    if shape == "Box":
        for gy in (range(-R, R + cy) if dim == 3 else [0]):
            segs.append((gy, -R, 2 * R + cx))
    else:
        if dim == 3:
            segs += [(gy, 0, cx) for gy in range(-R, 0)] + [(gy, 0, cx) for gy in range(cy, cy + R)]
        segs += [(gy, -R, 2 * R + cx) for gy in range(cy if dim == 3 else 1)]
    out = []
    for gy, gx0, n in segs:
        for i in range(n):
            if aligned(gx0 + i) and i + 1 < n:
                out.append((gx0 + i, gy))
    return out


def simulate(dim, shape, R, c, block, grid, left_offset, right_offset, aligned, es=8, smem_optin=232448,
             num_sms=148, occ=2, chunk=0, depth=0, nctas=0, orient="Row"):
    cx, cy = c[0], c[1] if dim == 3 else 1
    vec = 16 // es
    xdim, ydim = grid[0], grid[1]
    zdim = grid[2] if dim == 3 else 1
    ro = right_offset if aligned else 0
    x0 = R + left_offset
    x_lim, y_lim = xdim - R - ro, ydim - R
    z_lim = zdim - R if dim == 3 else 1
    bx, by = block[0], (block[1] if dim == 3 else 1)
    TX, TY = bx * cx, (by * cy if dim == 3 else 1)
    if TX % vec:
        return None
    rows = TY + 2 * R if dim == 3 else 1
    lshift = left_offset % vec
    if chunk:
        ch = chunk
    elif dim == 3:
        ch = 1
    else:
        want = max(1, min(16, cdiv(4096, (TX + 2 * R + vec) * es)))
        ch = 1
        while ch * 2 <= want:
            ch *= 2
    W = pipe_width(TX, R, lshift, vec, ch, rows, es)
    if rows > 256:  # wider rows than a TMA box stream through cp.async (single-grid sweeps)
        return None
    plane = W * rows
    CHUNK = ch * plane
    chunk_bytes = CHUNK * es
    assert chunk_bytes % 128 == 0
    d = depth or max(2, min(6, cdiv(24576, chunk_bytes)))
    while True:
        nslot = 1 + d
        smem = cdiv(nslot * 8, 128) * 128 + 128 + nslot * chunk_bytes
        if smem <= smem_optin or d == 1:
            break
        d -= 1
    if smem > smem_optin:
        return None
    ring_elems = nslot * CHUNK
    ex = max(0, x_lim - x0)
    ey = y_lim - R
    ntx = max(1, cdiv(ex, TX))
    nty, M = 1, ey
    if dim == 3:
        nty, M = max(1, cdiv(ey, TY)), z_lim - R
    total = ntx * nty * M
    n = nctas or num_sms * occ
    per = max(1, cdiv(total, n))
    gridb = max(1, cdiv(total, per))
    pts = in_plane_points(dim, "Box" if shape == "Box" else "Star", R, cx, cy)
    pairs = pair_loads(dim, shape, orient, R, cx, cy, lshift)
    pair_store = cx % 2 == 0 and (lshift + R) % 2 == 0
    written = {}
    for cta in range(gridb):
        ring = [None] * ring_elems
        slot_of = [None] * nslot
        gc = 0
        w = cta * per
        w_end = min(w + per, total)
        while w < w_end:
            tile, zs = w // M, w % M
            ze = min(M, zs + (w_end - w))
            w += ze - zs
            ms, nout = R + zs, ze - zs
            np_ = nout + 2 * R
            nch = cdiv(np_, ch)
            X0 = x0 + (tile % ntx) * TX
            xl = X0 - R - lshift
            assert xl >= 0 and xl % vec == 0, "TMA x coordinate not on a 16-byte granule"
            Y0 = R + (tile // ntx) * TY if dim == 3 else 0
            issued = set()

            def issue(j):
                slot = (gc + j) % nslot
                slot_of[slot] = gc + j
                issued.add(j)
                m0 = ms - R + j * ch
                base = slot * CHUNK
                assert base + CHUNK <= ring_elems
                for q in range(CHUNK):
                    xx = xl + q % W
                    if dim == 2:
                        yy = m0 + q // W
                        ring[base + q] = xx + yy * xdim if (xx < xdim and yy < ydim) else -1
                    else:
                        yy = Y0 - R + (q // W) % rows
                        zz = m0 + q // plane
                        ring[base + q] = (xx + yy * xdim + zz * xdim * ydim
                                          if (xx < xdim and yy < ydim and zz < zdim) else -1)

            for j in range(min(nslot - 1, nch)):
                issue(j)
            # the kernel's chunk loop with its slot cursor
            cur_slot, cur_par = gc % nslot, (gc // nslot) & 1
            for j in range(nch):
                assert cur_slot == (gc + j) % nslot and cur_par == ((gc + j) // nslot) & 1
                assert j in issued, "wait on a chunk never issued"
                assert slot_of[(gc + j) % nslot] == gc + j
                if j + nslot - 1 < nch:
                    # the slot being refilled held chunk j-1, consumed before the barrier
                    assert slot_of[(gc + j + nslot - 1) % nslot] in (None, gc + j - 1)
                    issue(j + nslot - 1)
                    assert slot_of[(gc + j) % nslot] == gc + j, "current chunk overwritten"
                for t in range(ch):
                    pi = j * ch + t
                    if pi >= np_:
                        continue
                    p = ms - R + pi
                    base = cur_slot * CHUNK + t * plane
                    op = pi - 2 * R
                    for ty in range(by):
                        for tx in range(bx):
                            x = X0 + tx * cx
                            col0 = lshift + R + tx * cx
                            if dim == 3:
                                y = Y0 + ty * cy
                                lane_off = (R + ty * cy) * W + col0
                                lane_ok = x + cx - 1 < x_lim and y + cy - 1 < y_lim
                            else:
                                y = 0
                                lane_off = col0
                                lane_ok = x + cx - 1 < x_lim
                            for gx, gy in pts:
                                idx = base + lane_off + gy * W + gx
                                assert 0 <= idx < ring_elems, "shared-memory read out of bounds"
                                if dim == 2:
                                    want = (x + gx) + p * xdim
                                else:
                                    want = (x + gx) + (y + gy) * xdim + p * xdim * ydim
                                if lane_ok:
                                    assert ring[idx] == want, "read %r want %r" % (ring[idx], want)
                            for gx, gy in pairs:
                                idx = base + lane_off + gy * W + gx
                                assert idx % 2 == 0 and idx + 1 < ring_elems, "pair load not aligned"
                            if lane_ok and 0 <= op < nout and pair_store and xdim % 2 == 0:
                                # the kernel's st_pair rule (base pointers are pair-aligned in the model)
                                for ey in range(cy):
                                    for ex_ in range(0, cx, 2):
                                        o0 = x + ex_ + ((y + ey) * xdim if dim == 3 else 0) + \
                                            (ms + op) * (xdim * ydim if dim == 3 else xdim)
                                        assert o0 % 2 == 0, "pair store not aligned"
                            if lane_ok and 0 <= op < nout:
                                for ey in range(cy):
                                    for ex_ in range(cx):
                                        if dim == 2:
                                            o = (x + ex_) + (ms + op) * xdim
                                        else:
                                            o = (x + ex_) + (y + ey) * xdim + (ms + op) * xdim * ydim
                                        written[o] = written.get(o, 0) + 1
                cur_slot += 1
                if cur_slot == nslot:
                    cur_slot, cur_par = 0, cur_par ^ 1
            gc += nch
    count = 0
    zr = range(R, z_lim) if dim == 3 else [0]
    for z in zr:
        for yy in range(R, y_lim):
            for xx in range(x0, x_lim):
                o = xx + yy * xdim + z * xdim * ydim
                assert written.get(o, 0) == 1, "interior point written %d times" % written.get(o, 0)
                count += 1
    assert len(written) == count, "a point outside the interior was written"
    return count


def batch_pieces(grids, total, per_cta):
    """Pieces of tcs_pipe_batch: grids = [(first, n_tiles, m)] ascending by first.

    Mirrors the kernel: a CTA's range [b*per, min((b+1)*per, total)) starts at the last grid
    whose first item is <= the range start (binary search), then walks pieces, each inside one
    tile of one grid.  Returns [(cta, grid, tile, zs, ze)]."""
    out = []
    ng = len(grids)
    nctas = max(1, -(-total // per_cta))
    for b in range(nctas):
        w0 = b * per_cta
        w1 = min(w0 + per_cta, total)
        lo, hi = 0, ng
        while hi - lo > 1:
            mid = (lo + hi) // 2
            if grids[mid][0] <= w0:
                lo = mid
            else:
                hi = mid
        gi = lo
        w = w0
        while w < w1:
            while gi + 1 < ng and grids[gi + 1][0] <= w:
                gi += 1
            first, _, m = grids[gi]
            local = w - first
            tile, zs = divmod(local, m)
            ze = min(m, zs + (w1 - w))
            w += ze - zs
            out.append((b, gi, tile, zs, ze))
    return out


def copy_chunk(dim, E, pw, rows, chp, xl, y0, m0, xdim, ydim, zdim):
    """Ring chunk filled by pipe_copy_chunk<E> (tcs_kernels.cuh): element offset -> global linear
    index, or -1 for a zero fill.  Asserts the alignment rules of the E-element copies."""
    out = {}
    nseg = pw // E
    assert pw % E == 0
    nrow = chp * rows if dim == 3 else chp
    for q in range(nrow * nseg):
        row = q // nseg
        xx = xl + (q - row * nseg) * E
        if dim == 2:
            yy, zz = m0 + row, 0
            inside = xx < xdim and yy < ydim
        else:
            t = row // rows
            yy, zz = y0 + row - t * rows, m0 + t
            inside = xx < xdim and yy < ydim and zz < zdim
        gi = xx + (yy + zz * ydim) * xdim if inside else 0
        if inside:
            assert gi % E == 0  # source aligned to the copy size (base aligned to it too)
            assert xx + E - 1 < xdim
        d = q * E
        for k in range(E):
            out[d + k] = gi + k if inside else -1
    return out
