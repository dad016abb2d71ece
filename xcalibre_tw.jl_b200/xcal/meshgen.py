"""Synthetic meshes for the benchmark and test configurations.

The 2D generators write I-DEAS universal files (datasets 2411 nodes, 2412
elements, 2467 groups) in the subset that the reference's loader reads
(src/UNV2/UNV2_1_loader.jl:3-120): boundary edges first, then quadrilaterals,
then one group per patch.  Both the library's mesh builder and the oracle read
these files, so the reference numbering of faces and cells is produced by the
reference's own construction rules.

The 3D generator (hexahedral cavity) builds the flattened mesh directly, as the
reference has no working 3D builder; it follows the 2D conventions: boundary
faces first, owner1 < owner2, normal from owner1 to owner2, boundary delta equal
to the full cell-to-face distance, weight as in src/UNV2/UNV2_2_geometry.jl:71,
cell volume from the divergence theorem (1/3 sum x_f . S_f in 3D).
"""
import math

import numpy as np


# ---------------------------------------------------------------- UNV writer
def write_unv(path, nodes, edges_by_patch, quads):
    """nodes: (n,3) float; edges_by_patch: list of (name, [(a,b),...]) with 1-based
    node ids; quads: (m,4) 1-based node ids, counter-clockwise."""
    lines = []
    ap = lines.append
    ap("    -1")
    ap("  2411")
    for i, (x, y, z) in enumerate(nodes):
        ap(f"{i + 1:10d}{1:10d}{1:10d}{11:10d}")
        ap(f"{x:25.16E}{y:25.16E}{z:25.16E}")
    ap("    -1")
    ap("    -1")
    ap("  2412")
    eid = 0
    group_elems = []
    for name, edges in edges_by_patch:
        ids = []
        for (a, b) in edges:
            eid += 1
            ap(f"{eid:10d}{11:10d}{2:10d}{1:10d}{7:10d}{2:10d}")
            ap(f"{0:10d}{1:10d}{1:10d}")
            ap(f"{a:10d}{b:10d}")
            ids.append(eid)
        group_elems.append((name, ids))
    for q in quads:
        eid += 1
        ap(f"{eid:10d}{44:10d}{2:10d}{1:10d}{7:10d}{4:10d}")
        ap(f"{q[0]:10d}{q[1]:10d}{q[2]:10d}{q[3]:10d}")
    ap("    -1")
    ap("    -1")
    ap("  2467")
    for g, (name, ids) in enumerate(group_elems):
        ap(f"{g + 1:10d}{0:10d}{0:10d}{0:10d}{0:10d}{0:10d}{0:10d}{len(ids):10d}")
        ap(name)
        for k in range(0, len(ids), 2):
            pair = ids[k:k + 2]
            ap("".join(f"{8:10d}{e:10d}{0:10d}{0:10d}" for e in pair))
    ap("    -1")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def _structured_block(xs, ys, node0):
    """Node ids of a structured block, row-major (x fastest), 1-based from node0+1."""
    nx, ny = len(xs), len(ys)
    return (node0 + 1 + np.arange(nx * ny)).reshape(ny, nx)


def cavity_unv(path, n=40, L=0.1):
    """Lid-driven cavity, n x n uniform quads on [0,L]^2 (patches inlet x=0,
    outlet x=L, bottom y=0, top y=L, the naming of the reference's quad40.unv)."""
    xs = np.linspace(0.0, L, n + 1)
    ys = np.linspace(0.0, L, n + 1)
    X, Y = np.meshgrid(xs, ys)
    nodes = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1)
    ids = _structured_block(xs, ys, 0)
    inlet = [(ids[j, 0], ids[j + 1, 0]) for j in range(n)]
    outlet = [(ids[j, n], ids[j + 1, n]) for j in range(n)]
    bottom = [(ids[0, i], ids[0, i + 1]) for i in range(n)]
    top = [(ids[n, i], ids[n, i + 1]) for i in range(n)]
    quads = [(ids[j, i], ids[j, i + 1], ids[j + 1, i + 1], ids[j + 1, i])
             for j in range(n) for i in range(n)]
    write_unv(path, nodes, [("inlet", inlet), ("outlet", outlet), ("bottom", bottom),
                            ("top", top)], quads)
    return dict(ncells=n * n)


def graded(n, length, ratio, both=True):
    """n intervals over [0,length], geometric growth `ratio` away from both ends
    (or from the start only), returned as n+1 monotone coordinates."""
    if both:
        h = n // 2
        w = ratio ** np.arange(h)
        w = np.concatenate([w, w[::-1]]) if n % 2 == 0 else np.concatenate([w, [w[-1] * ratio], w[::-1]])
    else:
        w = ratio ** np.arange(n)
    x = np.concatenate([[0.0], np.cumsum(w)])
    return x / x[-1] * length


def bfs_unv(path, h=0.01, cells_per_h=27, ratio=1.05, jitter=0.1, seed=20240101):
    """Laminar backward-facing step: inlet channel x in [-5h,0], y in [h,2h];
    outlet x in [0,30h], y in [0,2h]; y grading `ratio` toward the walls with
    matched node distributions on the block interface; interior nodes jittered
    by U(-jitter, jitter) x local spacing in x and y (boundary nodes fixed).
    Patches: inlet, outlet, wall, top (the reference's BFS naming)."""
    ch = cells_per_h
    nxi, nxo = 5 * ch, 30 * ch
    nyu = ch                      # cells across one step height
    yu = h + graded(nyu, h, ratio)          # upper half [h, 2h]
    yl = graded(nyu, h, ratio)              # lower half [0, h]
    y_out = np.concatenate([yl, yu[1:]])    # outlet block, 2*ch cells
    x_in = np.linspace(-5 * h, 0.0, nxi + 1)
    x_out = np.linspace(0.0, 30 * h, nxo + 1)
    # node grid: outlet block (nxo+1) x (2ch+1) plus inlet block nodes left of x=0
    nodes = []
    idx_out = np.zeros((2 * nyu + 1, nxo + 1), dtype=np.int64)
    idx_in = np.zeros((nyu + 1, nxi + 1), dtype=np.int64)
    for j, y in enumerate(y_out):
        for i, x in enumerate(x_out):
            nodes.append((x, y, 0.0))
            idx_out[j, i] = len(nodes)
    for j, y in enumerate(yu):
        for i, x in enumerate(x_in):
            if i == nxi:                     # x = 0 shared with the outlet block
                idx_in[j, i] = idx_out[nyu + j, 0]
                continue
            nodes.append((x, y, 0.0))
            idx_in[j, i] = len(nodes)
    nodes = np.array(nodes, dtype=np.float64)
    # boundary node flags
    rng = np.random.default_rng(seed)
    fixed = np.zeros(len(nodes) + 1, dtype=bool)
    inlet = [(idx_in[j, 0], idx_in[j + 1, 0]) for j in range(nyu)]
    outlet = [(idx_out[j, nxo], idx_out[j + 1, nxo]) for j in range(2 * nyu)]
    top = ([(idx_in[nyu, i], idx_in[nyu, i + 1]) for i in range(nxi)] +
           [(idx_out[2 * nyu, i], idx_out[2 * nyu, i + 1]) for i in range(nxo)])
    wall = ([(idx_in[0, i], idx_in[0, i + 1]) for i in range(nxi)] +          # step top y=h
            [(idx_out[j, 0], idx_out[j + 1, 0]) for j in range(nyu)] +       # step face x=0
            [(idx_out[0, i], idx_out[0, i + 1]) for i in range(nxo)])        # floor y=0
    for e in inlet + outlet + top + wall:
        fixed[e[0]] = fixed[e[1]] = True
    # jitter interior nodes by local spacing (mean of adjacent intervals)
    dx_in = x_in[1] - x_in[0]
    dx_out = x_out[1] - x_out[0]

    def local_dy(ys, j):
        a = ys[j] - ys[j - 1] if j > 0 else ys[1] - ys[0]
        b = ys[j + 1] - ys[j] if j + 1 < len(ys) else ys[-1] - ys[-2]
        return 0.5 * (a + b)
    shifts = {}
    for j in range(2 * nyu + 1):
        for i in range(nxo + 1):
            nid = idx_out[j, i]
            if not fixed[nid]:
                shifts[nid] = (dx_out, local_dy(y_out, j))
    for j in range(nyu + 1):
        for i in range(nxi):
            nid = idx_in[j, i]
            if not fixed[nid]:
                shifts[nid] = (dx_in, local_dy(yu, j))
    for nid in sorted(shifts):
        sx, sy = shifts[nid]
        u = rng.uniform(-jitter, jitter, size=2)
        nodes[nid - 1, 0] += u[0] * sx
        nodes[nid - 1, 1] += u[1] * sy
    quads = []
    for j in range(nyu):
        for i in range(nxi):
            quads.append((idx_in[j, i], idx_in[j, i + 1], idx_in[j + 1, i + 1], idx_in[j + 1, i]))
    for j in range(2 * nyu):
        for i in range(nxo):
            quads.append((idx_out[j, i], idx_out[j, i + 1], idx_out[j + 1, i + 1], idx_out[j + 1, i]))
    write_unv(path, nodes, [("inlet", inlet), ("outlet", outlet), ("wall", wall), ("top", top)], quads)
    return dict(ncells=len(quads))


def flatplate_unv(path, nx=600, ny=250, L=1.0, H=0.2, U=10.0, nu=1.5e-5, rx=1.02, ry=1.08):
    """k-omega flat plate, nx x ny quads on [0,L] x [0,H].  The growth ratios are
    read as maximum cell-to-cell ratios: y1 from y+ = 1 with the Schlichting
    skin-friction correlation at Re_L, grown by ry until the spacing reaches the
    uniform remainder; streamwise likewise from the leading edge with rx.
    Patches: inlet, outlet, wall, top."""
    ReL = U * L / nu
    cf = (2 * math.log10(ReL) - 0.65) ** -2.3
    utau = U * math.sqrt(cf / 2)
    y1 = nu / utau

    def stretch(n, length, d1, r):
        # spacing grows by r from d1 until it would exceed the uniform spacing of
        # the rest of the interval, then stays constant
        ds = [d1]
        while True:
            used = sum(ds)
            rem = length - used
            left = n - len(ds)
            if left <= 0:
                break
            nxt = ds[-1] * r
            if nxt * left >= rem:
                ds.extend([rem / left] * left)
                break
            ds.append(nxt)
        x = np.concatenate([[0.0], np.cumsum(ds)])
        return x / x[-1] * length
    ys = stretch(ny, H, y1, ry)
    xs = stretch(nx, L, L / nx * 0.1, rx)
    X, Y = np.meshgrid(xs, ys)
    nodes = np.stack([X.ravel(), Y.ravel(), np.zeros(X.size)], axis=1)
    ids = _structured_block(xs, ys, 0)
    inlet = [(ids[j, 0], ids[j + 1, 0]) for j in range(ny)]
    outlet = [(ids[j, nx], ids[j + 1, nx]) for j in range(ny)]
    wall = [(ids[0, i], ids[0, i + 1]) for i in range(nx)]
    top = [(ids[ny, i], ids[ny, i + 1]) for i in range(nx)]
    quads = [(ids[j, i], ids[j, i + 1], ids[j + 1, i + 1], ids[j + 1, i])
             for j in range(ny) for i in range(nx)]
    write_unv(path, nodes, [("inlet", inlet), ("outlet", outlet), ("wall", wall), ("top", top)], quads)
    return dict(ncells=nx * ny, y1=float(ys[1] - ys[0]))


# ------------------------------------------------------------ 3D hex cavity
def hex_cavity(n=128, L=1.0):
    """Uniform n^3 hexahedral cavity on [0,L]^3 in the flattened reference
    layout (1-based int64 indices).  Patches (in order): xmin, xmax, ymin, lid
    (y = L), zmin, zmax.  Returns a dict of numpy arrays."""
    h = L / n
    N = n * n * n
    ii, jj, kk = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    # cell id: i fastest (x), then j (y), then k (z)
    cid = (ii + n * jj + n * n * kk)
    cc = np.zeros((N, 3))
    cc[cid.ravel(), 0] = (ii.ravel() + 0.5) * h
    cc[cid.ravel(), 1] = (jj.ravel() + 0.5) * h
    cc[cid.ravel(), 2] = (kk.ravel() + 0.5) * h
    area = h * h
    faces_o1, faces_o2, fcent, fnorm = [], [], [], []
    patches = []
    # boundary faces, patch by patch
    for axis, side, name in ((0, 0, "xmin"), (0, 1, "xmax"), (1, 0, "ymin"), (1, 1, "lid"),
                             (2, 0, "zmin"), (2, 1, "zmax")):
        sel = [ii, jj, kk][axis] == (0 if side == 0 else n - 1)
        cells = np.sort(cid[sel].ravel())
        o = cells
        ctr = cc[o].copy()
        ctr[:, axis] = 0.0 if side == 0 else L
        nrm = np.zeros((len(o), 3))
        nrm[:, axis] = -1.0 if side == 0 else 1.0
        patches.append((name, o))
        faces_o1.append(o); faces_o2.append(o); fcent.append(ctr); fnorm.append(nrm)
    nbf = sum(len(p[1]) for p in patches)
    # internal faces: for each cell in id order, its +x, +y, +z neighbours
    o1_list, o2_list = [], []
    for axis, stride in ((0, 1), (1, n), (2, n * n)):
        coord = [ii, jj, kk][axis]
        sel = coord < n - 1
        a = cid[sel].ravel()
        o1_list.append(a); o2_list.append(a + stride)
    ia = np.concatenate(o1_list)
    ib = np.concatenate(o2_list)
    axis_of = np.concatenate([np.full(len(x), ax) for ax, x in enumerate(o1_list)])
    order = np.lexsort((ib, ia))          # internal faces sorted by (owner1, owner2)
    ia, ib, axis_of = ia[order], ib[order], axis_of[order]
    nfi = len(ia)
    ictr = 0.5 * (cc[ia] + cc[ib])
    inrm = np.zeros((nfi, 3))
    inrm[np.arange(nfi), axis_of] = 1.0
    o1 = np.concatenate(faces_o1 + [ia])
    o2 = np.concatenate(faces_o2 + [ib])
    fc = np.concatenate(fcent + [ictr])
    fn = np.concatenate(fnorm + [inrm])
    nf = len(o1)
    farea = np.full(nf, area)
    d12 = cc[o2] - cc[o1]
    delta = np.sqrt((d12[:, 0] * d12[:, 0] + d12[:, 1] * d12[:, 1]) + d12[:, 2] * d12[:, 2])
    dcf = fc[:nbf] - cc[o1[:nbf]]
    delta[:nbf] = np.sqrt((dcf[:, 0] * dcf[:, 0] + dcf[:, 1] * dcf[:, 1]) + dcf[:, 2] * dcf[:, 2])
    fe = np.zeros((nf, 3))
    fe[nbf:] = d12[nbf:] / delta[nbf:, None]
    fe[:nbf] = dcf / delta[:nbf, None]
    d1f = fc - cc[o1]
    df2 = cc[o2] - fc
    a1 = (d1f[:, 0] * fn[:, 0] + d1f[:, 1] * fn[:, 1]) + d1f[:, 2] * fn[:, 2]
    a2 = (df2[:, 0] * fn[:, 0] + df2[:, 1] * fn[:, 1]) + df2[:, 2] * fn[:, 2]
    weight = np.ones(nf)
    weight[nbf:] = np.abs(a1[nbf:] / (a1[nbf:] + a2[nbf:]))
    # per-cell internal face lists in face-id order
    fid = np.arange(nbf, nf)
    cells_of = np.concatenate([o1[nbf:], o2[nbf:]])
    faces_of = np.concatenate([fid, fid])
    nbr_of = np.concatenate([o2[nbf:], o1[nbf:]])
    sign_of = np.concatenate([np.ones(nfi, dtype=np.int64), -np.ones(nfi, dtype=np.int64)])
    order = np.lexsort((faces_of, cells_of))
    cells_of, faces_of, nbr_of, sign_of = cells_of[order], faces_of[order], nbr_of[order], sign_of[order]
    counts = np.bincount(cells_of, minlength=N)
    ptr = np.concatenate([[0], np.cumsum(counts)])
    # volume: 1/3 sum over internal faces ((d_cf.n)*nsign)*area, then boundary faces
    dcf_all = fc[faces_of] - cc[cells_of]
    contrib = (((dcf_all[:, 0] * fn[faces_of, 0] + dcf_all[:, 1] * fn[faces_of, 1])
                + dcf_all[:, 2] * fn[faces_of, 2]) * sign_of) * area
    vol = np.zeros(N)
    np.add.at(vol, cells_of, contrib)
    vol = vol / 3.0
    bcontrib = ((dcf[:, 0] * fn[:nbf, 0] + dcf[:, 1] * fn[:nbf, 1]) + dcf[:, 2] * fn[:nbf, 2]) / 3.0 * area
    np.add.at(vol, o1[:nbf], bcontrib)
    pptr = [0]
    pf, pc = [], []
    off = 0
    for name, cells in patches:
        pf.append(np.arange(off, off + len(cells)) + 1)
        pc.append(cells + 1)
        off += len(cells)
        pptr.append(off)
    return dict(
        ncells=N, nfaces=nf, nbfaces=nbf, dim=3,
        cell_centre=np.ascontiguousarray(cc.ravel()), cell_volume=vol,
        cell_faces_ptr=(ptr + 1).astype(np.int64), cell_faces=(faces_of + 1).astype(np.int64),
        cell_neighbours=(nbr_of + 1).astype(np.int64), cell_nsign=sign_of.astype(np.int64),
        face_owner=np.ascontiguousarray(np.stack([o1 + 1, o2 + 1], axis=1).ravel()).astype(np.int64),
        face_centre=np.ascontiguousarray(fc.ravel()), face_normal=np.ascontiguousarray(fn.ravel()),
        face_e=np.ascontiguousarray(fe.ravel()), face_area=farea, face_delta=delta,
        face_weight=weight, patch_names=[p[0] for p in patches],
        patch_ptr=np.array(pptr, dtype=np.int64), patch_faces=np.concatenate(pf).astype(np.int64),
        patch_cells=np.concatenate(pc).astype(np.int64))
