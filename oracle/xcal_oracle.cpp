// xcal_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Single-threaded FP64 CPU restatement of the reference's (TimW-24/XCALibre_TW.jl,
// module FVM_1D v0.2.0) 2D steady SIMPLE / transient PISO path, used as the
// parity checker for libxcal.so.  Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py load this library; the product
// never links or calls it.
//
// Every function cites the reference file:line it restates.  Choices where the
// reference's behaviour is not defined by its own sources:
//   * Krylov.jl 0.9.5 (not vendored) -- CG and BiCGSTAB are restated from the
//     package's published algorithm and documented conventions: warm start
//     (x0 enters through r0 = b - A*x0 and is added back at the end), stopping
//     test ||r|| <= atol + rtol*||r0|| measured on the preconditioned residual,
//     BiCGSTAB with left preconditioner M and shadow vector c = b, itmax.
//   * Reductions (BLAS dot/nrm2, Base.sum/mean) have no pinned order in the
//     reference (BLAS-implementation dependent).  Every reduction here uses the
//     project's canonical order (canon_sum below), which the device kernels
//     reproduce exactly; that makes the FP64 device path bitwise comparable.
//   * CG on the pressure system: the assembled p matrix is negative definite, for
//     which Krylov.jl's CG takes sqrt of a negative <r,z> and throws.  CG is run
//     on the negated system (-A)x = -b, which is mathematically the same solve;
//     negation is exact, so this equals flipping the sign of <r,z> and <p,Ap>.
//   * GMRES (Krylov.jl 0.9.5 gmres!, restart = false, left preconditioner M,
//     modified Gram-Schmidt, Givens QR via sym_givens (SymOrtho), back
//     substitution, x = V y) restated from the same published algorithm.
//   * ILU0 (ILUZero.jl 0.2.0, not vendored): ILU(0) in the IKJ form with L
//     entries scaled by the reciprocal of the pivot; ldiv! as unit-lower
//     forward substitution (ascending columns) and upper backward substitution
//     subtracting in descending column order before dividing by the diagonal
//     (the order of a column-oriented CSC sweep).
//   * DILU's O(n^2) upper_row_indices is built in O(nnz) with identical output.
//   * The "3D extension" (dim == 3): the reference is 2D-only; the same formulas
//     carried to the z component (uz equation, 3-component interpolation, H and
//     correction).  It has no reference counterpart.
// Parity against the reference's own Julia run is unpinned: Julia is not
// available, and the reference has no golden vectors for this path.
//
// Build: oracle/Makefile (g++ -O2 -ffp-contract=off: no FMA contraction).

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>
#include <set>
#include <map>
#include <algorithm>
#include <limits>
#include <chrono>

#include "../include/xcal.h"

typedef int64_t i64;

// ------------------------------------------------------------------ vectors
struct V3 { double x, y, z; };
static inline V3 v3(double a, double b, double c) { V3 r; r.x = a; r.y = b; r.z = c; return r; }
static inline V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline V3 vscale(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
static inline V3 vdiv(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }
// StaticArrays 1.9.1 dot: ((a1*b1 + a2*b2) + a3*b3)
static inline double vdot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
// StaticArrays 1.9.1 norm: sqrt((a1^2 + a2^2) + a3^2) (unscaled branch, 0<l<Inf)
static inline double vnorm(V3 a) { return std::sqrt((a.x * a.x + a.y * a.y) + a.z * a.z); }
// StaticArrays cross: (a2*b3-a3*b2, a3*b1-a1*b3, a1*b2-a2*b1)
static inline V3 vcross(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// Julia max(x::Float64, y::Float64): NaN-propagating, max(-0.0, 0.0) == 0.0
static inline double jmax(double a, double b) {
  if (a != a || b != b) return a + b;
  if (a > b) return a;
  if (b > a) return b;
  return std::signbit(a) ? b : a;
}

// ------------------------------------------------------- canonical reduction
// Fixed-tree sum: tiles of 256 values (one per lane); inside a tile a warp
// shuffle-down tree (offsets 16,8,4,2,1) then an 8-way tree over the warps.
// Tile partials are folded the same way (lane t sums partials t, t+256, ...
// sequentially, then the same tree).  The device reductions follow this order.
static double canon_tree256(double *w) {
  double ws[8];
  for (int wp = 0; wp < 8; ++wp) {
    double l[32];
    for (int i = 0; i < 32; ++i) l[i] = w[wp * 32 + i];
    for (int off = 16; off >= 1; off >>= 1)
      for (int i = 0; i < off; ++i) l[i] = l[i] + l[i + off];
    ws[wp] = l[0];
  }
  for (int off = 4; off >= 1; off >>= 1)
    for (int i = 0; i < off; ++i) ws[i] = ws[i] + ws[i + off];
  return ws[0];
}

template <class F>
static double canon_sum_f(i64 n, F f) {
  i64 ntiles = (n + 255) / 256;
  std::vector<double> part(ntiles);
  double w[256];
  for (i64 t = 0; t < ntiles; ++t) {
    for (int l = 0; l < 256; ++l) {
      i64 e = t * 256 + l;
      w[l] = (e < n) ? f(e) : 0.0;
    }
    part[t] = canon_tree256(w);
  }
  for (int l = 0; l < 256; ++l) {
    double s = (l < ntiles) ? part[l] : 0.0;
    for (i64 k = l + 256; k < ntiles; k += 256) s = s + part[k];
    w[l] = s;
  }
  return canon_tree256(w);
}
static double cdot(const std::vector<double> &x, const std::vector<double> &y) {
  return canon_sum_f((i64)x.size(), [&](i64 i) { return x[i] * y[i]; });
}
static double cnrm2(const std::vector<double> &x) { return std::sqrt(cdot(x, x)); }

// ----------------------------------------------------------------- mesh
struct OPatch { std::string name; std::vector<i64> faces, cells; };
struct OMesh {
  i64 nc = 0, nf = 0, nbf = 0;
  int dim = 2;
  std::vector<V3> ccentre; std::vector<double> cvol;
  std::vector<i64> cf_ptr, cf_face, cf_nbr, cf_sign;       // 0-based
  std::vector<i64> o1, o2;
  std::vector<V3> fcentre, fnormal, fe;
  std::vector<double> farea, fdelta, fweight;
  std::vector<OPatch> patches;
  i64 nnodes = 0;
  // export buffers (1-based, reference layout)
  std::vector<i64> x_cfp, x_cf, x_cn, x_cs, x_own, x_pptr, x_pf, x_pc;
  std::vector<double> x_cc, x_fc, x_fn, x_fe;
  std::string names;
};

// ---- UNV loader: src/UNV2/UNV2_1_loader.jl:3-120
struct UElem { i64 index, vcount; std::vector<i64> v; };
struct UBnd { std::string name; i64 group; std::vector<i64> elements; };

static bool parse_i64(const std::string &s, i64 &out) {
  if (s.empty()) return false;
  char *end = nullptr;
  errno = 0;
  long long v = strtoll(s.c_str(), &end, 10);
  if (*end != '\0' || errno) return false;
  out = v;
  return true;
}

static int unv_load(const char *path, std::vector<V3> &points, std::vector<UElem> &elements,
                    std::vector<UBnd> &bnds, std::string &err) {
  std::ifstream in(path);
  if (!in) { err = std::string("cannot open ") + path; return XCAL_ERR_IO; }
  bool blockStart = false, p2411 = false, p2412 = false, p2467 = false;
  i64 index = 0, vertexCount = 0;
  int currentBC = -1;
  std::string line;
  while (std::getline(in, line)) {
    std::istringstream ss(line);
    std::vector<std::string> s;
    std::string tok;
    while (ss >> tok) s.push_back(tok);
    if (s.empty()) continue;
    if (!blockStart && s[0] == "-1") { blockStart = true; continue; }
    if (blockStart && s[0] == "-1") { blockStart = false; p2411 = p2412 = p2467 = false; continue; }
    if (blockStart && s[0] == "2411" && !p2411 && !p2412 && !p2467) { p2411 = true; continue; }
    if (blockStart && s[0] == "2412" && !p2411 && !p2412 && !p2467) { p2412 = true; continue; }
    if (blockStart && s[0] == "2467" && !p2411 && !p2412 && !p2467) { p2467 = true; continue; }
    if (p2411) {
      if (s[0].find('.') != std::string::npos) {   // length(split(sline[1], ".")) > 1
        if (s.size() < 3) { err = "bad node line"; return XCAL_ERR_MESH; }
        points.push_back(v3(strtod(s[0].c_str(), nullptr), strtod(s[1].c_str(), nullptr),
                            strtod(s[2].c_str(), nullptr)));
        continue;
      }
    }
    if (p2412) {
      i64 first;
      if (!parse_i64(s[0], first)) { err = "bad element line"; return XCAL_ERR_MESH; }
      if (first == 0) continue;
      i64 last = 0;
      bool lastok = parse_i64(s.back(), last);
      if (s.size() == 6 && lastok && last == 2) { vertexCount = last; index = first; continue; }
      if (s.size() == 2) {
        UElem e; e.index = index; e.vcount = vertexCount;
        for (auto &t : s) { i64 v; parse_i64(t, v); e.v.push_back(v); }
        elements.push_back(e); continue;
      }
      if (s.size() == 6 && lastok && last == 3) { vertexCount = last; index = first; continue; }
      if (s.size() == 3) {
        UElem e; e.index = index; e.vcount = vertexCount;
        for (auto &t : s) { i64 v; parse_i64(t, v); e.v.push_back(v); }
        elements.push_back(e); continue;
      }
      if (s.size() == 6 && lastok && last == 4) { vertexCount = last; index = first; continue; }
      if (s.size() == 4) {
        UElem e; e.index = index; e.vcount = vertexCount;
        for (auto &t : s) { i64 v; parse_i64(t, v); e.v.push_back(v); }
        elements.push_back(e); continue;
      }
    }
    if (p2467) {
      i64 a, b;
      if (parse_i64(s[0], a) && s.size() > 1 && parse_i64(s[1], b) && b == 0) {
        UBnd nb; nb.name = "default"; nb.group = 0;
        bnds.push_back(nb);
        currentBC += 1;
        bnds[currentBC].group = currentBC + 1;
        continue;
      }
      if (!parse_i64(s[0], a)) {
        if (currentBC < 0) { err = "group name before group header"; return XCAL_ERR_MESH; }
        bnds[currentBC].name = s[0];
        continue;
      }
      if (currentBC < 0 || s.size() < 2) { err = "bad group entity line"; return XCAL_ERR_MESH; }
      i64 e1; parse_i64(s[1], e1);
      bnds[currentBC].elements.push_back(e1);
      if (s.size() >= 6) { i64 e2; parse_i64(s[5], e2); bnds[currentBC].elements.push_back(e2); }
    }
  }
  return XCAL_OK;
}

// ---- build_mesh: src/UNV2/UNV2_3_builder.jl:3-288, UNV2_2_geometry.jl:11-165
struct BFace { i64 n1, n2, o1, o2; V3 centre, normal, e; double area, delta, weight; };
struct BCell { std::vector<i64> nodes, faces, nbrs, nsign; V3 centre; double volume; };

static V3 geometric_centre(const std::vector<V3> &nodes, const i64 *ids, size_t n) {
  // UNV2_2_geometry.jl:11-18: sum starting at 0, divided by the count
  V3 s = v3(0.0, 0.0, 0.0);
  for (size_t i = 0; i < n; ++i) s = vadd(s, nodes[ids[i]]);
  return vdiv(s, (double)n);
}

static int build_mesh_unv(const char *path, double scale, OMesh &M, std::string &err) {
  std::vector<V3> points; std::vector<UElem> elements; std::vector<UBnd> bl;
  int st = unv_load(path, points, elements, bl, err);
  if (st) return st;
  if (scale != 1.0)   // scalePoints!, UNV2_3_builder.jl:48-54
    for (auto &p : points) p = vscale(p, scale);
  i64 bfaces = 0;       // total_boundary_faces(boundaryElements), :56-62
  for (auto &b : bl) bfaces += (i64)b.elements.size();
  i64 first = -1;       // first_2d_element, :64-73
  for (size_t i = 0; i < elements.size(); ++i) if (elements[i].vcount > 2) { first = (i64)i; break; }
  if (first < 0) { err = "no 2D elements"; return XCAL_ERR_MESH; }
  i64 np = (i64)points.size();
  // generate_nodes :77-91 (0-based node/cell ids)
  std::vector<std::vector<i64>> nodeCells(np);
  i64 cellID = 0;
  for (size_t i = first; i < elements.size(); ++i) {
    for (i64 nid : elements[i].v) {
      if (nid < 1 || nid > np) { err = "element references missing node"; return XCAL_ERR_MESH; }
      nodeCells[nid - 1].push_back(cellID);
    }
    cellID++;
  }
  // generate_faces :93-163: boundary faces first, then cell edges, then unique!
  std::vector<std::pair<i64, i64>> fn;
  for (auto &b : bl)
    for (i64 ei : b.elements) {
      if (ei < 1 || ei > (i64)elements.size() || elements[ei - 1].v.size() < 2) {
        err = "boundary element out of range"; return XCAL_ERR_MESH;
      }
      i64 a = elements[ei - 1].v[0], c = elements[ei - 1].v[1];
      if (a < c) fn.push_back({a, c});
      else if (a > c) fn.push_back({c, a});
      else { err = "Boundary elements are inconsistent: possible mesh corruption"; return XCAL_ERR_MESH; }
    }
  for (size_t i = first; i < elements.size(); ++i) {
    const auto &vv = elements[i].v;
    size_t nv = vv.size();
    for (size_t vi = 0; vi < nv; ++vi) {
      i64 a = vv[vi], c = (vi + 1 >= nv) ? vv[0] : vv[vi + 1];
      if (a < c) fn.push_back({a, c});
      else if (a > c) fn.push_back({c, a});
      else { err = "Boundary elements are inconsistent: possible mesh corruption"; return XCAL_ERR_MESH; }
    }
  }
  {  // unique! keeps the first occurrence, preserving order
    std::set<std::pair<i64, i64>> seen;
    std::vector<std::pair<i64, i64>> u;
    for (auto &f : fn) if (seen.insert(f).second) u.push_back(f);
    fn.swap(u);
  }
  i64 nf = (i64)fn.size();
  std::vector<BFace> faces(nf);
  for (i64 f = 0; f < nf; ++f) {
    faces[f].n1 = fn[f].first - 1; faces[f].n2 = fn[f].second - 1;
    faces[f].o1 = faces[f].o2 = -1;
    faces[f].area = faces[f].delta = faces[f].weight = 0.0;
    faces[f].centre = faces[f].normal = faces[f].e = v3(0, 0, 0);
  }
  // generate_cells :165-178
  i64 nc = (i64)elements.size() - first;
  std::vector<BCell> cells(nc);
  for (i64 c = 0; c < nc; ++c) {
    for (i64 nid : elements[first + c].v) cells[c].nodes.push_back(nid - 1);
    cells[c].volume = 0.0; cells[c].centre = v3(0, 0, 0);
  }
  // generate_boundaries :180-196
  std::vector<OPatch> patches;
  std::vector<std::vector<std::pair<i64, i64>>> pnodes;
  for (auto &b : bl) {
    OPatch p; p.name = b.name;
    std::vector<std::pair<i64, i64>> pn;
    for (i64 ei : b.elements) {
      i64 a = elements[ei - 1].v[0], c = elements[ei - 1].v[1];
      pn.push_back({std::min(a, c), std::max(a, c)});   // sort!(faceNodesID), :246
    }
    patches.push_back(p); pnodes.push_back(pn);
  }
  // face_cell_connectivity! :200-236
  for (i64 f = 0; f < nf; ++f) {
    i64 own[2] = {-1, -1};
    int cnt = 0;
    for (i64 c1 : nodeCells[faces[f].n1])
      for (i64 c2 : nodeCells[faces[f].n2])
        if (c1 == c2) {
          if (cnt >= 2) { err = "face shared by more than two cells"; return XCAL_ERR_MESH; }
          own[cnt++] = c1;
        }
    if (cnt == 0) { err = "face without owner cell"; return XCAL_ERR_MESH; }
    if (own[1] >= 0) {
      faces[f].o1 = own[0]; faces[f].o2 = own[1];
      cells[own[0]].faces.push_back(f); cells[own[1]].faces.push_back(f);
      cells[own[0]].nbrs.push_back(own[1]); cells[own[1]].nbrs.push_back(own[0]);
    } else {
      faces[f].o1 = own[0]; faces[f].o2 = own[0];
    }
  }
  // boundary_connectivity! :238-266 (searches faces 1..bfaces)
  for (size_t b = 0; b < patches.size(); ++b)
    for (auto &nd : pnodes[b])
      for (i64 f = 0; f < bfaces && f < nf; ++f)
        if (faces[f].n1 == nd.first - 1 && faces[f].n2 == nd.second - 1) {
          patches[b].faces.push_back(f);
          patches[b].cells.push_back(faces[f].o1);
        }
  // process_geometry! :39-44 -- centres
  std::vector<V3> nodes = points;
  for (auto &c : cells) c.centre = geometric_centre(nodes, c.nodes.data(), c.nodes.size());
  for (auto &f : faces) { i64 ids[2] = {f.n1, f.n2}; f.centre = geometric_centre(nodes, ids, 2); }
  // geometry! UNV2_2_geometry.jl:20-26
  i64 nbf = 0;
  for (auto &p : patches) nbf += (i64)p.faces.size();
  const V3 kk = v3(0.0, 0.0, 1.0);
  for (i64 f = nbf; f < nf; ++f) {   // internal_face_properties! :39-81
    BFace &fc = faces[f];
    V3 tangent = vsub(nodes[fc.n2], nodes[fc.n1]);
    double area = vnorm(tangent);
    V3 c1 = cells[fc.o1].centre, c2 = cells[fc.o2].centre, cf = fc.centre;
    V3 d_1f = vsub(cf, c1), d_f2 = vsub(c2, cf), d_12 = vsub(c2, c1);
    V3 ut = vdiv(tangent, area);
    V3 normal = vcross(ut, kk);
    if (vdot(d_12, normal) < 0.0) normal = vscale(normal, -1.0);
    double delta = vnorm(d_12);
    V3 e = vdiv(d_12, delta);
    double weight = std::fabs(vdot(d_1f, normal) / (vdot(d_1f, normal) + vdot(d_f2, normal)));
    fc.area = area; fc.normal = normal; fc.delta = delta; fc.e = e; fc.weight = weight;
  }
  for (auto &p : patches)   // boundary_face_properties! :84-120
    for (i64 f : p.faces) {
      BFace &fc = faces[f];
      V3 tangent = vsub(nodes[fc.n2], nodes[fc.n1]);
      double area = vnorm(tangent);
      V3 ut = vdiv(tangent, area);
      V3 normal = vcross(ut, kk);
      V3 d_cf = vsub(fc.centre, cells[fc.o1].centre);
      if (vdot(d_cf, normal) < 0.0) normal = vscale(normal, -1.0);
      double delta = vnorm(d_cf);
      fc.area = area; fc.normal = normal; fc.delta = delta; fc.e = vdiv(d_cf, delta); fc.weight = 1.0;
    }
  for (auto &c : cells) {   // cell_properties! :122-147
    double volume = 0.0;
    for (i64 f : c.faces) {
      V3 d_cf = vsub(faces[f].centre, c.centre);
      i64 s = (vdot(d_cf, faces[f].normal) > 0.0) ? 1 : -1;
      c.nsign.push_back(s);
      volume += (vdot(d_cf, faces[f].normal) * (double)s) * faces[f].area;
      c.volume = 0.5 * volume;
    }
  }
  for (auto &p : patches)   // correct_boundary_cell_volumes! :149-165
    for (size_t i = 0; i < p.cells.size(); ++i) {
      BCell &c = cells[p.cells[i]];
      const BFace &fc = faces[p.faces[i]];
      V3 d_cf = vsub(fc.centre, c.centre);
      c.volume = c.volume + (0.5 * vdot(d_cf, fc.normal)) * fc.area;
    }
  // update_mesh_format: src/Mesh/Mesh2D/Mesh2D_0_update_mesh.jl:5-142
  M.nc = nc; M.nf = nf; M.nbf = nbf; M.dim = 2; M.nnodes = np;
  M.ccentre.resize(nc); M.cvol.resize(nc); M.cf_ptr.assign(nc + 1, 0);
  for (i64 c = 0; c < nc; ++c) {
    M.ccentre[c] = cells[c].centre; M.cvol[c] = cells[c].volume;
    M.cf_ptr[c + 1] = M.cf_ptr[c] + (i64)cells[c].faces.size();
    for (size_t j = 0; j < cells[c].faces.size(); ++j) {
      M.cf_face.push_back(cells[c].faces[j]); M.cf_nbr.push_back(cells[c].nbrs[j]);
      M.cf_sign.push_back(cells[c].nsign[j]);
    }
  }
  M.o1.resize(nf); M.o2.resize(nf); M.fcentre.resize(nf); M.fnormal.resize(nf); M.fe.resize(nf);
  M.farea.resize(nf); M.fdelta.resize(nf); M.fweight.resize(nf);
  for (i64 f = 0; f < nf; ++f) {
    M.o1[f] = faces[f].o1; M.o2[f] = faces[f].o2; M.fcentre[f] = faces[f].centre;
    M.fnormal[f] = faces[f].normal; M.fe[f] = faces[f].e; M.farea[f] = faces[f].area;
    M.fdelta[f] = faces[f].delta; M.fweight[f] = faces[f].weight;
  }
  M.patches = patches;
  return XCAL_OK;
}

static int mesh_from_desc(const xcal_mesh_desc *d, OMesh &M, std::string &err) {
  if (!d || d->ncells <= 0 || d->nfaces <= 0 || d->nbfaces < 0 || d->nbfaces > d->nfaces) {
    err = "bad mesh counts"; return XCAL_ERR_ARG;
  }
  M.nc = d->ncells; M.nf = d->nfaces; M.nbf = d->nbfaces; M.dim = d->dim == 3 ? 3 : 2;
  i64 nc = M.nc, nf = M.nf;
  M.ccentre.resize(nc); M.cvol.resize(nc);
  for (i64 c = 0; c < nc; ++c) {
    M.ccentre[c] = v3(d->cell_centre[3 * c], d->cell_centre[3 * c + 1], d->cell_centre[3 * c + 2]);
    M.cvol[c] = d->cell_volume[c];
  }
  M.cf_ptr.resize(nc + 1);
  for (i64 c = 0; c <= nc; ++c) M.cf_ptr[c] = d->cell_faces_ptr[c] - 1;
  i64 tot = M.cf_ptr[nc];
  if (M.cf_ptr[0] != 0 || tot < 0) { err = "bad cell_faces_ptr"; return XCAL_ERR_MESH; }
  M.cf_face.resize(tot); M.cf_nbr.resize(tot); M.cf_sign.resize(tot);
  for (i64 k = 0; k < tot; ++k) {
    M.cf_face[k] = d->cell_faces[k] - 1; M.cf_nbr[k] = d->cell_neighbours[k] - 1;
    M.cf_sign[k] = d->cell_nsign[k];
    if (M.cf_face[k] < 0 || M.cf_face[k] >= nf || M.cf_nbr[k] < 0 || M.cf_nbr[k] >= nc) {
      err = "cell face list out of range"; return XCAL_ERR_MESH;
    }
  }
  M.o1.resize(nf); M.o2.resize(nf); M.fcentre.resize(nf); M.fnormal.resize(nf); M.fe.resize(nf);
  M.farea.resize(nf); M.fdelta.resize(nf); M.fweight.resize(nf);
  for (i64 f = 0; f < nf; ++f) {
    M.o1[f] = d->face_owner[2 * f] - 1; M.o2[f] = d->face_owner[2 * f + 1] - 1;
    if (M.o1[f] < 0 || M.o1[f] >= nc || M.o2[f] < 0 || M.o2[f] >= nc) { err = "owner out of range"; return XCAL_ERR_MESH; }
    M.fcentre[f] = v3(d->face_centre[3 * f], d->face_centre[3 * f + 1], d->face_centre[3 * f + 2]);
    M.fnormal[f] = v3(d->face_normal[3 * f], d->face_normal[3 * f + 1], d->face_normal[3 * f + 2]);
    M.fe[f] = v3(d->face_e[3 * f], d->face_e[3 * f + 1], d->face_e[3 * f + 2]);
    M.farea[f] = d->face_area[f]; M.fdelta[f] = d->face_delta[f]; M.fweight[f] = d->face_weight[f];
  }
  M.patches.resize(d->npatches);
  for (i64 p = 0; p < d->npatches; ++p) {
    M.patches[p].name = "patch" + std::to_string(p);
    for (i64 k = d->patch_ptr[p]; k < d->patch_ptr[p + 1]; ++k) {
      M.patches[p].faces.push_back(d->patch_faces[k] - 1);
      M.patches[p].cells.push_back(d->patch_cells[k] - 1);
    }
  }
  return XCAL_OK;
}

static void mesh_export_prepare(OMesh &M) {
  i64 nc = M.nc, nf = M.nf;
  M.x_cfp.resize(nc + 1);
  for (i64 c = 0; c <= nc; ++c) M.x_cfp[c] = M.cf_ptr[c] + 1;
  i64 tot = M.cf_ptr[nc];
  M.x_cf.resize(tot); M.x_cn.resize(tot); M.x_cs.resize(tot);
  for (i64 k = 0; k < tot; ++k) { M.x_cf[k] = M.cf_face[k] + 1; M.x_cn[k] = M.cf_nbr[k] + 1; M.x_cs[k] = M.cf_sign[k]; }
  M.x_own.resize(2 * nf);
  M.x_fc.resize(3 * nf); M.x_fn.resize(3 * nf); M.x_fe.resize(3 * nf);
  for (i64 f = 0; f < nf; ++f) {
    M.x_own[2 * f] = M.o1[f] + 1; M.x_own[2 * f + 1] = M.o2[f] + 1;
    M.x_fc[3 * f] = M.fcentre[f].x; M.x_fc[3 * f + 1] = M.fcentre[f].y; M.x_fc[3 * f + 2] = M.fcentre[f].z;
    M.x_fn[3 * f] = M.fnormal[f].x; M.x_fn[3 * f + 1] = M.fnormal[f].y; M.x_fn[3 * f + 2] = M.fnormal[f].z;
    M.x_fe[3 * f] = M.fe[f].x; M.x_fe[3 * f + 1] = M.fe[f].y; M.x_fe[3 * f + 2] = M.fe[f].z;
  }
  M.x_cc.resize(3 * nc);
  for (i64 c = 0; c < nc; ++c) { M.x_cc[3 * c] = M.ccentre[c].x; M.x_cc[3 * c + 1] = M.ccentre[c].y; M.x_cc[3 * c + 2] = M.ccentre[c].z; }
  M.x_pptr.assign(M.patches.size() + 1, 0);
  M.x_pf.clear(); M.x_pc.clear(); M.names.clear();
  for (size_t p = 0; p < M.patches.size(); ++p) {
    for (size_t k = 0; k < M.patches[p].faces.size(); ++k) {
      M.x_pf.push_back(M.patches[p].faces[k] + 1); M.x_pc.push_back(M.patches[p].cells[k] + 1);
    }
    M.x_pptr[p + 1] = (i64)M.x_pf.size();
    M.names += M.patches[p].name; M.names += "\n";
  }
}

// ---------------------------------------------------------- sparse matrix
// Equation(mesh): sparse(i, j, v) of sparse_matrix_connectivity,
// src/ModelFramework/ModelFramework_0_types.jl:90-125.  CSC, rows sorted,
// duplicate (i,j) merged.
struct CSC {
  i64 n = 0;
  std::vector<i64> colptr, rowval;
  std::vector<double> nzval;
  double get(i64 r, i64 c) const {
    for (i64 p = colptr[c]; p < colptr[c + 1]; ++p) if (rowval[p] == r) return nzval[p];
    return 0.0;
  }
  i64 pos(i64 r, i64 c) const {
    for (i64 p = colptr[c]; p < colptr[c + 1]; ++p) if (rowval[p] == r) return p;
    return -1;
  }
};

static void build_pattern(const OMesh &M, CSC &A) {
  i64 n = M.nc;
  std::vector<std::vector<i64>> colrows(n);
  for (i64 c = 0; c < n; ++c) {
    colrows[c].push_back(c);                                    // (cID, cID)
    for (i64 k = M.cf_ptr[c]; k < M.cf_ptr[c + 1]; ++k) colrows[M.cf_nbr[k]].push_back(c);  // (cID, nbr)
  }
  A.n = n; A.colptr.assign(n + 1, 0); A.rowval.clear();
  for (i64 c = 0; c < n; ++c) {
    auto &r = colrows[c];
    std::sort(r.begin(), r.end());
    r.erase(std::unique(r.begin(), r.end()), r.end());
    for (i64 x : r) A.rowval.push_back(x);
    A.colptr[c + 1] = (i64)A.rowval.size();
  }
  A.nzval.assign(A.rowval.size(), 0.0);
}

// mul!(y, A, x) for SparseMatrixCSC (SparseArrays, Julia 1.10): y=0, column scatter
static void spmv(const CSC &A, const std::vector<double> &x, std::vector<double> &y) {
  std::fill(y.begin(), y.end(), 0.0);
  for (i64 j = 0; j < A.n; ++j) {
    double xj = x[j];
    for (i64 p = A.colptr[j]; p < A.colptr[j + 1]; ++p) y[A.rowval[p]] += A.nzval[p] * xj;
  }
}

// ------------------------------------------------------------ preconditioners
// src/Solve/Preconditioners/preconditioners_0_types.jl, _1_DILU.jl, _2_functions.jl
struct Precon {
  int type = XCAL_PRECON_DILU;
  const CSC *A = nullptr;
  std::vector<double> D;            // DILU: inverse pivots after update; Jacobi/NormDiag: scale
  std::vector<i64> Di;
  std::vector<std::vector<i64>> Ri, J;
  // ILU(0): CSR view of the pattern (ascending columns), its CSC positions,
  // diagonal positions and the factor values (L strictly lower, U upper)
  std::vector<i64> rp, cl, cpos, dp;
  std::vector<double> F;
  i64 find(i64 r, i64 c) const {
    for (i64 e = rp[r]; e < rp[r + 1]; ++e) {
      if (cl[e] == c) return e;
      if (cl[e] > c) break;
    }
    return -1;
  }
  void setup(int t, const CSC *Am) {
    type = t; A = Am;
    i64 n = A->n;
    D.assign(n, 0.0);
    if (type == XCAL_PRECON_ILU0) {
      rp.assign(n + 1, 0);
      for (i64 j = 0; j < n; ++j) for (i64 p = A->colptr[j]; p < A->colptr[j + 1]; ++p) rp[A->rowval[p] + 1]++;
      for (i64 i = 0; i < n; ++i) rp[i + 1] += rp[i];
      cl.assign(rp[n], 0); cpos.assign(rp[n], 0); dp.assign(n, -1);
      std::vector<i64> fill(rp.begin(), rp.end() - 1);
      for (i64 j = 0; j < n; ++j)
        for (i64 p = A->colptr[j]; p < A->colptr[j + 1]; ++p) {
          i64 r = A->rowval[p], e = fill[r]++;
          cl[e] = j; cpos[e] = p;
          if (r == j) dp[r] = e;
        }
      F.assign(rp[n], 0.0);
      return;
    }
    if (type != XCAL_PRECON_DILU) return;
    Di.assign(n, 0);   // diagonal_indices! :159-174
    i64 idx = 0;
    for (i64 i = 0; i < n; ++i) {
      for (i64 p = A->colptr[i]; p < A->colptr[i + 1]; ++p) if (A->rowval[p] == i) { idx = p; break; }
      Di[i] = idx;
    }
    // upper_row_indices :178-200, built in O(nnz) with the same output
    Ri.assign(n, {}); J.assign(n, {});
    for (i64 j = 0; j < n; ++j)
      for (i64 p = A->colptr[j]; p <= Di[j]; ++p) {
        i64 row = A->rowval[p];
        if (row < j) { Ri[row].push_back(p); J[row].push_back(j); }
      }
  }
  void update() {   // update_preconditioner!
    const CSC &a = *A;
    i64 n = a.n;
    if (type == XCAL_PRECON_DILU) {   // update_dilu_diagonal! :202-251 (Algo 3)
      for (i64 i = 0; i < n; ++i) D[i] = a.nzval[Di[i]];
      for (i64 i = 0; i < n; ++i) {
        i64 c_start = Di[i] + 1, c_end = a.colptr[i + 1] - 1;
        i64 r_count = 0;
        for (i64 cp = c_start; cp <= c_end; ++cp) {
          i64 j = a.rowval[cp];
          D[j] -= a.nzval[cp] * a.nzval[Ri[i][r_count]] / D[i];
          r_count++;
        }
        D[i] = 1 / D[i];
      }
    } else if (type == XCAL_PRECON_ILU0) {   // ilu0!(P.storage, P.A), preconditioners_2_functions.jl:59-65
      for (size_t e = 0; e < F.size(); ++e) F[e] = a.nzval[cpos[e]];
      for (i64 i = 0; i < n; ++i)
        for (i64 e = rp[i]; e < rp[i + 1]; ++e) {
          i64 k = cl[e];
          if (k >= i) break;
          const double l = F[e] * (1.0 / F[dp[k]]);
          F[e] = l;
          for (i64 m = e + 1; m < rp[i + 1]; ++m) {
            i64 pos = find(k, cl[m]);
            if (pos >= 0) F[m] = F[m] - l * F[pos];
          }
        }
    } else if (type == XCAL_PRECON_JACOBI) {   // preconditioners_2_functions.jl:43-57
      for (i64 i = 0; i < n; ++i) D[i] = 1 / std::fabs(a.nzval[a.pos(i, i)]);
    } else if (type == XCAL_PRECON_NORMDIAG) {   // :28-41
      for (i64 i = 0; i < n; ++i) {
        double s = 0.0;
        for (i64 p = a.colptr[i]; p < a.colptr[i + 1]; ++p) s += a.nzval[p] * a.nzval[p];
        D[i] = 1 / std::sqrt(s);
      }
    }
  }
  // y = M^{-1} v  (LinearOperator wrapping ldiv!, preconditioners_0_types.jl:134-146)
  void apply(const std::vector<double> &b, std::vector<double> &x) const {
    const CSC &a = *A;
    i64 n = a.n;
    if (type == XCAL_PRECON_DILU) {
      for (i64 i = 0; i < n; ++i) x[i] = b[i];    // forward_substitution! :253-279
      for (i64 j = 0; j < n; ++j)
        for (i64 cp = Di[j] + 1; cp <= a.colptr[j + 1] - 1; ++cp) {
          i64 i = a.rowval[cp];
          x[i] -= a.nzval[cp] * x[j] * D[j];
        }
      for (i64 i = 0; i < n; ++i) x[i] = x[i] * D[i];   // backward_substitution! :281-308
      for (i64 i = n - 2; i >= 0; --i)
        for (size_t pi = 0; pi < Ri[i].size(); ++pi)
          x[i] -= a.nzval[Ri[i][pi]] * x[J[i][pi]] * D[i];
    } else if (type == XCAL_PRECON_ILU0) {   // ldiv!(y, LU, v)
      std::vector<double> y(n);
      for (i64 i = 0; i < n; ++i) {
        double v = b[i];
        for (i64 e = rp[i]; e < rp[i + 1] && cl[e] < i; ++e) v = v - F[e] * y[cl[e]];
        y[i] = v;
      }
      for (i64 i = n - 1; i >= 0; --i) {
        double v = y[i];
        for (i64 e = rp[i + 1] - 1; e >= rp[i] && cl[e] > i; --e) v = v - F[e] * x[cl[e]];
        x[i] = v / F[dp[i]];
      }
    } else if (type == XCAL_PRECON_NONE) {
      for (i64 i = 0; i < n; ++i) x[i] = b[i];
    } else {
      for (i64 i = 0; i < n; ++i) x[i] = D[i] * b[i];   // opDiagonal
    }
  }
};

// ----------------------------------------------------------------- Krylov
// Krylov.jl 0.9.5 semantics (see file header).  Returns the iteration count.
static int krylov_cg(const CSC &A, const std::vector<double> &b, std::vector<double> &values,
                     const Precon &M, int itmax, double atol, double rtol, double *rnorm_out) {
  i64 n = A.n;
  std::vector<double> dx = values, x(n, 0.0), r(n), z(n), p(n), Ap(n);
  spmv(A, dx, r);                                        // mul!(r, A, Δx)
  for (i64 i = 0; i < n; ++i) r[i] = b[i] - r[i];        // @kaxpby!(n, 1, b, -1, r)
  M.apply(r, z);
  p = z;
  double gamma = cdot(r, z);
  double sgn = (gamma < 0.0) ? -1.0 : 1.0;               // negated-system formulation
  gamma = sgn * gamma;
  double rNorm = std::sqrt(gamma);
  int iter = 0;
  if (gamma == 0.0) {
    for (i64 i = 0; i < n; ++i) values[i] = x[i] + dx[i];
    if (rnorm_out) *rnorm_out = rNorm;
    return 0;
  }
  const double eps = std::numeric_limits<double>::epsilon();
  double pNorm2 = gamma;
  double epsl = atol + rtol * rNorm;
  bool solved = rNorm <= epsl, tired = iter >= itmax, zero_curv = false;
  while (!(solved || tired || zero_curv)) {
    spmv(A, p, Ap);
    double pAp = sgn * cdot(p, Ap);
    if (pAp <= eps * pNorm2 && std::fabs(pAp) <= eps * pNorm2) { zero_curv = true; continue; }
    double alpha = gamma / pAp;
    for (i64 i = 0; i < n; ++i) x[i] = x[i] + alpha * p[i];
    for (i64 i = 0; i < n; ++i) r[i] = r[i] + (-alpha) * Ap[i];
    M.apply(r, z);
    double gnext = sgn * cdot(r, z);
    rNorm = std::sqrt(gnext);
    bool mach = (rNorm + 1.0 <= 1.0);
    solved = (rNorm <= epsl) || mach;
    if (!solved) {
      double beta = gnext / gamma;
      pNorm2 = gnext + (beta * beta) * pNorm2;
      gamma = gnext;
      for (i64 i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    iter++;
    tired = iter >= itmax;
  }
  for (i64 i = 0; i < n; ++i) values[i] = x[i] + dx[i];
  if (rnorm_out) *rnorm_out = rNorm;
  return iter;
}

static int krylov_bicgstab(const CSC &A, const std::vector<double> &b, std::vector<double> &values,
                           const Precon &M, int itmax, double atol, double rtol, double *rnorm_out) {
  i64 n = A.n;
  std::vector<double> dx = values, x(n, 0.0), s(n, 0.0), v(n, 0.0), r0(n), r(n), p(n), q(n), t(n);
  spmv(A, dx, r0);
  for (i64 i = 0; i < n; ++i) r0[i] = b[i] - r0[i];
  M.apply(r0, r);
  p = r;
  double rho = 1.0, alpha = 1.0, omega = 1.0;
  (void)rho;
  double rNorm = cnrm2(r);
  int iter = 0;
  if (rNorm == 0.0) {
    for (i64 i = 0; i < n; ++i) values[i] = x[i] + dx[i];
    if (rnorm_out) *rnorm_out = rNorm;
    return 0;
  }
  double epsl = atol + rtol * rNorm;
  const std::vector<double> &c = b;
  double next_rho = cdot(c, r);
  if (next_rho == 0.0) {
    for (i64 i = 0; i < n; ++i) values[i] = x[i] + dx[i];
    if (rnorm_out) *rnorm_out = rNorm;
    return 0;
  }
  bool solved = rNorm <= epsl, tired = iter >= itmax, breakdown = false;
  while (!(solved || tired || breakdown)) {
    iter++;
    rho = next_rho;
    spmv(A, p, q);                                                   // q = A*y (y = p)
    M.apply(q, v);                                                   // v = M^{-1} q
    alpha = rho / cdot(c, v);
    for (i64 i = 0; i < n; ++i) s[i] = r[i] + (-alpha) * v[i];       // s = r - alpha*v
    for (i64 i = 0; i < n; ++i) x[i] = x[i] + alpha * p[i];
    spmv(A, s, q);                                                   // d = A*z (z = s)
    M.apply(q, t);                                                   // t = M^{-1} d
    omega = cdot(t, s) / cdot(t, t);
    for (i64 i = 0; i < n; ++i) x[i] = x[i] + omega * s[i];
    for (i64 i = 0; i < n; ++i) r[i] = s[i] + (-omega) * t[i];       // r = s - omega*t
    next_rho = cdot(c, r);
    double beta = (next_rho / rho) * (alpha / omega);
    for (i64 i = 0; i < n; ++i) p[i] = p[i] + (-omega) * v[i];
    for (i64 i = 0; i < n; ++i) p[i] = r[i] + beta * p[i];
    rNorm = cnrm2(r);
    bool mach = (rNorm + 1.0 <= 1.0);
    solved = (rNorm <= epsl) || mach;
    tired = iter >= itmax;
    breakdown = (alpha == 0.0 || std::isnan(alpha));
  }
  for (i64 i = 0; i < n; ++i) values[i] = x[i] + dx[i];
  if (rnorm_out) *rnorm_out = rNorm;
  return iter;
}

// SymOrtho plane rotation (Choi, Paige & Saunders), Krylov.jl sym_givens
static void sym_givens(double a, double b, double &c, double &s, double &rho) {
  auto sgn = [](double v) { return v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : v); };
  if (b == 0.0) {
    c = (a == 0.0) ? 1.0 : sgn(a);
    s = 0.0;
    rho = std::fabs(a);
  } else if (a == 0.0) {
    c = 0.0;
    s = sgn(b);
    rho = std::fabs(b);
  } else if (std::fabs(b) > std::fabs(a)) {
    double t = a / b;
    s = sgn(b) / std::sqrt(1.0 + t * t);
    c = s * t;
    rho = b / s;
  } else {
    double t = b / a;
    c = sgn(a) / std::sqrt(1.0 + t * t);
    s = c * t;
    rho = a / c;
  }
}

// gmres! (restart = false, reorthogonalization = false, N = I)
static int krylov_gmres(const CSC &A, const std::vector<double> &b, std::vector<double> &values,
                        const Precon &M, int itmax, double atol, double rtol, double *rnorm_out) {
  i64 n = A.n;
  std::vector<double> dx = values, x(n, 0.0), w(n), r0(n), q(n);
  spmv(A, dx, w);
  for (i64 i = 0; i < n; ++i) w[i] = b[i] - w[i];        // w = b - A*Δx
  M.apply(w, r0);                                          // r0 = M w
  double beta = cnrm2(r0), rNorm = beta;
  const double btol = 1.8189894035458565e-12;             // eps^(3/4) = 2^-39
  int iter = 0;
  if (beta == 0.0) {
    for (i64 i = 0; i < n; ++i) values[i] = x[i] + dx[i];
    if (rnorm_out) *rnorm_out = rNorm;
    return 0;
  }
  double epsl = atol + rtol * rNorm;
  bool solved = rNorm <= epsl, tired = iter >= itmax;
  if (!(solved || tired)) {
    std::vector<std::vector<double>> V(1, std::vector<double>(n));
    std::vector<double> R, c, s, z(1, beta);
    for (i64 i = 0; i < n; ++i) V[0][i] = r0[i] / rNorm;
    int k = 0;
    bool inner_tired = false, breakdown = false;
    size_t nr = 0;
    while (!(solved || inner_tired || breakdown)) {
      ++k;
      R.resize(nr + k, 0.0); c.resize(k, 0.0); s.resize(k, 0.0);
      spmv(A, V[k - 1], w);
      M.apply(w, q);
      for (int i = 0; i < k; ++i) {                        // modified Gram-Schmidt
        R[nr + i] = cdot(V[i], q);
        for (i64 j = 0; j < n; ++j) q[j] = q[j] + (-R[nr + i]) * V[i][j];
      }
      double Hbis = cnrm2(q);
      for (int i = 0; i < k - 1; ++i) {
        double tmp = c[i] * R[nr + i] + s[i] * R[nr + i + 1];
        R[nr + i + 1] = s[i] * R[nr + i] - c[i] * R[nr + i + 1];
        R[nr + i] = tmp;
      }
      sym_givens(R[nr + k - 1], Hbis, c[k - 1], s[k - 1], R[nr + k - 1]);
      double zeta = s[k - 1] * z[k - 1];
      z[k - 1] = c[k - 1] * z[k - 1];
      rNorm = std::fabs(zeta);
      nr += k;
      iter++;
      bool mach = (rNorm + 1.0 <= 1.0);
      solved = (rNorm <= epsl) || mach;
      breakdown = Hbis <= btol;
      inner_tired = k >= itmax;
      if (!(solved || inner_tired || breakdown)) {
        V.emplace_back(n);
        for (i64 i = 0; i < n; ++i) V[k][i] = q[i] / Hbis;
        z.push_back(zeta);
      }
    }
    std::vector<double> y(z.begin(), z.begin() + k);       // back substitution R y = z
    for (int i = k - 1; i >= 0; --i) {
      for (int j = k - 1; j >= i + 1; --j) y[i] = y[i] - R[(size_t)j * (j + 1) / 2 + i] * y[j];
      double rii = R[(size_t)i * (i + 1) / 2 + i];
      y[i] = (std::fabs(rii) <= btol) ? 0.0 : y[i] / rii;
    }
    for (int i = 0; i < k; ++i)
      for (i64 j = 0; j < n; ++j) x[j] = x[j] + y[i] * V[i][j];
  }
  for (i64 i = 0; i < n; ++i) values[i] = x[i] + dx[i];
  if (rnorm_out) *rnorm_out = rNorm;
  return iter;
}

static int krylov_solve(int solver, const CSC &A, const std::vector<double> &b, std::vector<double> &x,
                        const Precon &M, int itmax, double atol, double rtol, double *rn) {
  if (solver == XCAL_SOLVER_CG) return krylov_cg(A, b, x, M, itmax, atol, rtol, rn);
  if (solver == XCAL_SOLVER_GMRES) return krylov_gmres(A, b, x, M, itmax, atol, rtol, rn);
  return krylov_bicgstab(A, b, x, M, itmax, atol, rtol, rn);
}

// ------------------------------------------------------------- equations
// Model terms in declaration order (Time, Divergence, Laplacian, Si) and sources:
// src/ModelFramework/ModelFramework_1_operations.jl:3-58
struct Terms {
  bool has_time = false; int time = XCAL_TIME_STEADY; double dt = 1.0;
  bool has_div = false; int div = XCAL_DIV_UPWIND; const std::vector<double> *mdot = nullptr;
  bool has_lap = false; int lap_sign = 1; const std::vector<double> *gamma = nullptr;
  bool has_si = false; const std::vector<double> *si = nullptr;   // cell field, sign +1
  int nsrc = 0; const std::vector<double> *src[2] = {nullptr, nullptr}; int src_sign[2] = {1, 1};
  const std::vector<double> *phi = nullptr;   // field being solved (Si wall BC)
};

struct Eqn { CSC A; std::vector<double> b; };

// _discretise!: src/Discretise/Discretise_2_generated_distretisation.jl:5-81 with the
// per-term scheme!/scheme_source! of src/Discretise/Discretise_1_schemes.jl:11-113
static void discretise(const OMesh &M, Eqn &E, const Terms &T, const std::vector<double> &prev) {
  CSC &A = E.A;
  std::fill(A.nzval.begin(), A.nzval.end(), 0.0);
  i64 cIndex = 0;
  for (i64 c = 0; c < M.nc; ++c) {
    for (i64 k = M.cf_ptr[c]; k < M.cf_ptr[c + 1]; ++k) {
      i64 f = M.cf_face[k], nID = M.cf_nbr[k];
      double ns = (double)M.cf_sign[k];
      cIndex = A.pos(c, c);
      i64 nIndex = A.pos(c, nID);
      if (T.has_div) {
        if (T.div == XCAL_DIV_UPWIND) {           // :258-266
          double ap = 1.0 * ((*T.mdot)[f] * ns);
          A.nzval[cIndex] += jmax(ap, 0.0);
          A.nzval[nIndex] += -jmax(-ap, 0.0);
        } else {                                  // :238-251
          V3 xf = M.fcentre[f], xC = M.ccentre[c], xN = M.ccentre[nID];
          double weight = vnorm(vsub(xf, xC)) / vnorm(vsub(xN, xC));
          double omw = 1.0 - weight;
          double ap = 1.0 * ((*T.mdot)[f] * ns);
          A.nzval[cIndex] += ap * omw;
          A.nzval[nIndex] += ap * weight;
        }
      }
      if (T.has_lap) {                            // :221-229
        double ap = (double)T.lap_sign * ((-(*T.gamma)[f]) * M.farea[f]) / M.fdelta[f];
        A.nzval[cIndex] += ap;
        A.nzval[nIndex] += -ap;
      }
    }
    if (M.cf_ptr[c + 1] == M.cf_ptr[c]) cIndex = A.pos(c, c);  // (reference leaves cIndex stale here)
    E.b[c] = 0.0;
    double volume = M.cvol[c];
    if (T.has_time && T.time == XCAL_TIME_EULER) {   // :204-217
      double rdt = 1 / T.dt;
      A.nzval[cIndex] += volume * rdt;
      E.b[c] += prev[c] * volume * rdt;
    }
    if (T.has_si) {                                  // :283-294
      double flux = 1.0 * (*T.si)[c] * volume;
      A.nzval[cIndex] += flux;
    }
    for (int s = 0; s < T.nsrc; ++s)                 // generated block 3, :32-37
      E.b[c] += (double)T.src_sign[s] * (*T.src[s])[c] * volume;
  }
}

// _apply_boundary_conditions!: src/Discretise/Discretise_4_apply_bcs.jl:7-44 with the
// functors of src/Discretise/Discretise_3_boundary_conditions.jl:4-160.  comp selects
// the vector component of the BC value.
static void apply_bcs(const OMesh &M, Eqn &E, const Terms &T, const std::vector<xcal_bc> &bcs, int comp) {
  CSC &A = E.A;
  for (const xcal_bc &bc : bcs) {
    const OPatch &P = M.patches[bc.patch];
    double value = bc.value[comp];
    for (size_t i = 0; i < P.cells.size(); ++i) {
      i64 f = P.faces[i], c = P.cells[i];
      i64 d = A.pos(c, c);
      if (T.has_div) {
        double ap = 1.0 * (*T.mdot)[f];
        if (T.div == XCAL_DIV_UPWIND) {
          if (bc.type == XCAL_BC_DIRICHLET) E.b[c] -= ap * value;                    // :164-178
          else if (bc.type == XCAL_BC_NEUMANN || bc.type == XCAL_BC_KWALL || bc.type == XCAL_BC_OMEGAWALL)
            A.nzval[d] += jmax(ap, 0.0);                                             // :180-209
        } else {
          if (bc.type == XCAL_BC_DIRICHLET) E.b[c] += 1.0 * ((-(*T.mdot)[f]) * value);   // :132-138
          else if (bc.type == XCAL_BC_NEUMANN || bc.type == XCAL_BC_KWALL || bc.type == XCAL_BC_OMEGAWALL)
            A.nzval[d] += ap;                                                        // :140-162
        }
      }
      if (T.has_lap && bc.type == XCAL_BC_DIRICHLET) {                               // :94-105
        double flux = (*T.gamma)[f] * M.farea[f] / M.fdelta[f];
        double ap = (double)T.lap_sign * (-flux);
        A.nzval[d] += ap;
        E.b[c] += ap * value;
      }
      if (T.has_si && bc.type == XCAL_BC_OMEGAWALL) {                                // :234-241
        double phi = (*T.phi)[c];
        double flux = 1.0 * (*T.si)[c];
        E.b[c] += flux * phi * M.cvol[c];
      }
    }
  }
}

// Generic model equation (a user-built Model of operators and sources, as
// ModelFramework_1_operations.jl:3-58 builds it): _discretise! with the terms
// in model order (src/Discretise/Discretise_2_generated_distretisation.jl:5-81,
// scheme!/scheme_source! of Discretise_1_schemes.jl:11-113), then
// _apply_boundary_conditions! (Discretise_4_apply_bcs.jl:7-44, functors of
// Discretise_3_boundary_conditions.jl:4-241) when bcs are given.  Face fields
// are per face, cell fields per cell, in the mesh's own numbering.
static void discretise_terms(const OMesh &M, Eqn &E, const xcal_term *terms, int nterms, const xcal_source *srcs,
                             int nsrc, const double *prev, double dt) {
  CSC &A = E.A;
  std::fill(A.nzval.begin(), A.nzval.end(), 0.0);
  i64 cIndex = 0;
  for (i64 c = 0; c < M.nc; ++c) {
    for (i64 k = M.cf_ptr[c]; k < M.cf_ptr[c + 1]; ++k) {
      const i64 f = M.cf_face[k], nID = M.cf_nbr[k];
      const double ns = (double)M.cf_sign[k];
      cIndex = A.pos(c, c);
      const i64 nIndex = A.pos(c, nID);
      for (int t = 0; t < nterms; ++t) {
        const xcal_term &T = terms[t];
        if (T.kind == XCAL_TERM_LAPLACIAN) {
          const double ap = T.sign * (-T.flux[f] * M.farea[f]) / M.fdelta[f];
          A.nzval[cIndex] += ap;
          A.nzval[nIndex] += -ap;
        } else if (T.kind == XCAL_TERM_DIVERGENCE && T.scheme == XCAL_DIV_LINEAR) {
          const V3 xf = M.fcentre[f], xC = M.ccentre[c], xN = M.ccentre[nID];
          const double weight = vnorm(vsub(xf, xC)) / vnorm(vsub(xN, xC));
          const double omw = 1.0 - weight;
          const double ap = T.sign * (T.flux[f] * ns);
          A.nzval[cIndex] += ap * omw;
          A.nzval[nIndex] += ap * weight;
        } else if (T.kind == XCAL_TERM_DIVERGENCE) {
          const double ap = T.sign * (T.flux[f] * ns);
          A.nzval[cIndex] += jmax(ap, 0.0);
          A.nzval[nIndex] += -jmax(-ap, 0.0);
        }
      }
    }
    if (M.cf_ptr[c + 1] == M.cf_ptr[c]) cIndex = A.pos(c, c);
    E.b[c] = 0.0;
    const double volume = M.cvol[c];
    for (int t = 0; t < nterms; ++t) {
      const xcal_term &T = terms[t];
      if (T.kind == XCAL_TERM_TIME && T.scheme == XCAL_TIME_EULER) {
        const double rdt = 1 / dt;
        A.nzval[cIndex] += volume * rdt;
        E.b[c] += prev[c] * volume * rdt;
      } else if (T.kind == XCAL_TERM_SI) {
        const double flux = T.sign * T.flux[c] * volume;
        A.nzval[cIndex] += flux;
      }
    }
    for (int q = 0; q < nsrc; ++q) E.b[c] += srcs[q].sign * srcs[q].field[c] * volume;
  }
}

static void apply_bcs_terms(const OMesh &M, Eqn &E, const xcal_term *terms, int nterms, const xcal_bc *bcs, int nbc,
                            const double *phi, int comp) {
  CSC &A = E.A;
  for (int q = 0; q < nbc; ++q) {
    const xcal_bc &bc = bcs[q];
    const OPatch &P = M.patches[bc.patch];
    const double value = bc.value[comp];
    const bool wall = bc.type == XCAL_BC_NEUMANN || bc.type == XCAL_BC_KWALL || bc.type == XCAL_BC_OMEGAWALL;
    for (size_t i = 0; i < P.cells.size(); ++i) {
      const i64 f = P.faces[i], c = P.cells[i];
      const i64 d = A.pos(c, c);
      for (int t = 0; t < nterms; ++t) {
        const xcal_term &T = terms[t];
        if (T.kind == XCAL_TERM_LAPLACIAN) {
          if (bc.type == XCAL_BC_DIRICHLET) {
            const double flux = T.flux[f] * M.farea[f] / M.fdelta[f];
            const double ap = T.sign * (-flux);
            A.nzval[d] += ap;
            E.b[c] += ap * value;
          }
        } else if (T.kind == XCAL_TERM_DIVERGENCE && T.scheme == XCAL_DIV_LINEAR) {
          if (bc.type == XCAL_BC_DIRICHLET) E.b[c] += T.sign * (-T.flux[f] * value);
          else if (wall) A.nzval[d] += T.sign * (T.flux[f]);
        } else if (T.kind == XCAL_TERM_DIVERGENCE) {
          const double ap = T.sign * (T.flux[f]);
          if (bc.type == XCAL_BC_DIRICHLET) E.b[c] -= ap * value;
          else if (wall) A.nzval[d] += jmax(ap, 0.0);
        } else if (T.kind == XCAL_TERM_SI && bc.type == XCAL_BC_OMEGAWALL) {
          const double flux = T.sign * T.flux[c];
          E.b[c] += flux * phi[c] * M.cvol[c];
        }
      }
    }
  }
}

// implicit_relaxation!, setReference!, explicit_relaxation!: src/Solve/Solve_1_api.jl:48-68
static void implicit_relaxation(Eqn &E, const std::vector<double> &field, double alpha) {
  for (i64 i = 0; i < E.A.n; ++i) {
    i64 d = E.A.pos(i, i);
    E.A.nzval[d] /= alpha;
    E.b[i] += (1.0 - alpha) * E.A.nzval[d] * field[i];
  }
}
static void set_reference(Eqn &E, bool has, double pref, i64 cell) {
  if (!has) return;
  i64 d = E.A.pos(cell, cell);
  E.b[cell] += E.A.nzval[d] * pref;
  E.A.nzval[d] += E.A.nzval[d];
}
static void explicit_relaxation(std::vector<double> &phi, const std::vector<double> &phi0, double a) {
  for (size_t i = 0; i < phi.size(); ++i) phi[i] = phi0[i] + a * (phi[i] - phi0[i]);
}

// residual!: src/Solvers/Solvers_0_functions.jl:13-63
static double residual(const Eqn &E, const std::vector<double> &x) {
  i64 n = E.A.n;
  std::vector<double> Fx(n);
  spmv(E.A, x, Fx);
  double sR = canon_sum_f(n, [&](i64 i) { double d = std::fabs(Fx[i] - E.b[i]); return d * d; });
  double mean = sR / (double)n;
  double nb = cnrm2(E.b);
  return std::sqrt(mean) / nb;
}

// ----------------------------------------------------------- field kernels
typedef std::vector<double> Vec;

// interpolate! scalar/vector: src/Calculate/Calculate_2_interpolation.jl:112-148
static void interpolate_s(const OMesh &M, Vec &phif, const Vec &phi) {
  for (i64 f = 0; f < M.nf; ++f) {
    double w = M.fweight[f];
    double omw = 1.0 - w;
    phif[f] = w * phi[M.o1[f]] + omw * phi[M.o2[f]];
  }
}
static void interpolate_v(const OMesh &M, Vec *Uf, Vec *const *U, int ncomp) {
  for (i64 f = 0; f < M.nf; ++f) {
    double w = M.fweight[f];
    double omw = 1.0 - w;
    for (int d = 0; d < ncomp; ++d) Uf[d][f] = w * (*U[d])[M.o1[f]] + omw * (*U[d])[M.o2[f]];
  }
}
// interpolate_midpoint!: src/Calculate/Calculate_0_gradient.jl:116-144
static void interpolate_midpoint_s(const OMesh &M, Vec &phif, const Vec &phi) {
  for (i64 f = 0; f < M.nf; ++f) phif[f] = 0.5 * (phi[M.o1[f]] + phi[M.o2[f]]);
}
// correct_boundaries!/adjust_boundary!: Calculate_2_interpolation.jl:6-110
static void correct_boundaries_s(const OMesh &M, Vec &phif, const Vec &phi, const std::vector<xcal_bc> &bcs) {
  for (const xcal_bc &bc : bcs) {
    const OPatch &P = M.patches[bc.patch];
    for (size_t i = 0; i < P.faces.size(); ++i)
      phif[P.faces[i]] = (bc.type == XCAL_BC_DIRICHLET) ? bc.value[0] : phi[P.cells[i]];
  }
}
static void correct_boundaries_v(const OMesh &M, Vec *Uf, Vec *const *U, const std::vector<xcal_bc> &bcs) {
  for (const xcal_bc &bc : bcs) {
    const OPatch &P = M.patches[bc.patch];
    for (size_t i = 0; i < P.faces.size(); ++i)
      for (int d = 0; d < 3; ++d)
        Uf[d][P.faces[i]] = (bc.type == XCAL_BC_DIRICHLET) ? bc.value[d] : (*U[d])[P.cells[i]];
  }
}
// green_gauss!: src/Calculate/Calculate_1_green_gauss.jl:2-39
static void green_gauss(const OMesh &M, Vec &dx, Vec &dy, Vec &dz, const Vec &phif) {
  for (i64 c = 0; c < M.nc; ++c) {
    double rx = 0.0, ry = 0.0, rz = 0.0;
    for (i64 k = M.cf_ptr[c]; k < M.cf_ptr[c + 1]; ++k) {
      i64 f = M.cf_face[k];
      double ns = (double)M.cf_sign[k];
      double a = M.farea[f];
      V3 n = M.fnormal[f];
      rx += phif[f] * ((a * n.x) * ns);
      ry += phif[f] * ((a * n.y) * ns);
      rz += phif[f] * ((a * n.z) * ns);
    }
    double vol = M.cvol[c];
    dx[c] = rx / vol; dy[c] = ry / vol; dz[c] = rz / vol;
  }
  for (i64 f = 0; f < M.nbf; ++f) {
    i64 c = M.o1[f];
    double vol = M.cvol[c], a = M.farea[f];
    V3 n = M.fnormal[f];
    double bx = phif[f] * (a * n.x), by = phif[f] * (a * n.y), bz = phif[f] * (a * n.z);
    bx /= vol; by /= vol; bz /= vol;
    dx[c] += bx; dy[c] += by; dz[c] += bz;
  }
}
// correct_interpolation!: Calculate_0_gradient.jl:146-173
static void correct_interpolation(const OMesh &M, const Vec &dx, const Vec &dy, const Vec &dz,
                                  Vec &phif, const Vec &phi) {
  const double w = 0.5;
  for (i64 f = M.nbf; f < M.nf; ++f) {
    i64 a = M.o1[f], b = M.o2[f];
    double phifp = w * (phi[a] + phi[b]);
    V3 g = v3(w * (dx[a] + dx[b]), w * (dy[a] + dy[b]), w * (dz[a] + dz[b]));
    V3 rP = M.ccentre[a], rN = M.ccentre[b], rf = M.fcentre[f];
    V3 Ri = vsub(rf, v3(w * (rP.x + rN.x), w * (rP.y + rN.y), w * (rP.z + rN.z)));
    phif[f] = phifp + vdot(g, Ri);
  }
}
// grad! scalar (Orthogonal :96-104, Midpoint :175-183)
static void grad_scalar(const OMesh &M, int scheme, Vec &dx, Vec &dy, Vec &dz, Vec &phif,
                        const Vec &phi, const std::vector<xcal_bc> &bcs) {
  if (scheme == XCAL_GRAD_MIDPOINT) {
    interpolate_midpoint_s(M, phif, phi);
    correct_boundaries_s(M, phif, phi, bcs);
    green_gauss(M, dx, dy, dz, phif);
    for (int i = 0; i < 2; ++i) {
      correct_interpolation(M, dx, dy, dz, phif, phi);
      green_gauss(M, dx, dy, dz, phif);
    }
  } else {
    interpolate_s(M, phif, phi);
    correct_boundaries_s(M, phif, phi, bcs);
    green_gauss(M, dx, dy, dz, phif);
  }
}
// div!: src/Calculate/Calculate_0_divergence.jl:75-107
static void divergence(const OMesh &M, Vec &out, Vec *const Uf) {
  for (i64 c = 0; c < M.nc; ++c) {
    double vol = M.cvol[c];
    out[c] = 0.0;
    for (i64 k = M.cf_ptr[c]; k < M.cf_ptr[c + 1]; ++k) {
      i64 f = M.cf_face[k];
      double a = M.farea[f];
      V3 Sf = v3(a * M.fnormal[f].x, a * M.fnormal[f].y, a * M.fnormal[f].z);
      V3 u = v3(Uf[0][f], Uf[1][f], Uf[2][f]);
      out[c] += vdot(u, Sf) * (double)M.cf_sign[k] / vol;
    }
  }
  for (i64 f = 0; f < M.nbf; ++f) {
    i64 c = M.o1[f];
    double vol = M.cvol[c], a = M.farea[f];
    V3 Sf = v3(a * M.fnormal[f].x, a * M.fnormal[f].y, a * M.fnormal[f].z);
    V3 u = v3(Uf[0][f], Uf[1][f], Uf[2][f]);
    out[c] += vdot(u, Sf) / vol;
  }
}
// flux!: src/Solvers/Solvers_0_functions.jl:65-73
static void flux(const OMesh &M, Vec &mdot, Vec *const Uf) {
  for (i64 f = 0; f < M.nf; ++f) {
    double a = M.farea[f];
    V3 Sf = v3(a * M.fnormal[f].x, a * M.fnormal[f].y, a * M.fnormal[f].z);
    mdot[f] = vdot(v3(Uf[0][f], Uf[1][f], Uf[2][f]), Sf);
  }
}

// ---------------------------------------------------------- k-omega model
// src/RANSModels/RANSModels_kOmega.jl:114-415, RANSModels_functions.jl:5-88
struct KOmegaState {
  Vec kf, wf, nutf, nueffk, nueffw, Dkf, Dwf, Pk, Pw;
  Vec gxx, gyx, gzx, gxy, gyy, gzy, gxz, gyz, gzz;   // gradU tensor (Grad{S}(U).result)
  Eqn keq, weq; Precon Pkp, Pwp;
};

static double ylam_of(double E, double kappa) {   // y_plus_laminar :322-325
  double yL = 11.0;
  for (int i = 0; i < 10; ++i) yL = std::log(jmax(yL * E, 1.0)) / kappa;
  return yL;
}
static double nut_wall(double nu, double yplus, double kappa, double E) {   // :342-344
  return jmax(nu * (yplus * kappa / std::log(jmax(E * yplus, 1.0 + 1e-4)) - 1), 0.0);
}

// bound!: RANSModels_functions.jl:96-123 (sequential; later cells see updated values)
static void bound_field(const OMesh &M, Vec &field, double bnd) {
  const double eps = std::numeric_limits<double>::epsilon();
  for (i64 i = 0; i < M.nc; ++i) {
    double sum_flux = 0.0;
    i64 sum_area = 0;
    for (i64 k = M.cf_ptr[i]; k < M.cf_ptr[i + 1]; ++k) {
      sum_flux += jmax(field[M.cf_nbr[k]], eps);
      sum_area += 1;
    }
    double average = sum_flux / (double)sum_area;
    field[i] = jmax(jmax(field[i], average * (std::signbit(field[i]) ? 1.0 : 0.0)), bnd);
  }
}

// ------------------------------------------------------------ SIMPLE / PISO
struct Run {
  const OMesh *M; const xcal_case *cfg;
  std::vector<xcal_bc> bcU, bcp, bck, bcw, bcn;
};

static double g_last_loop_seconds = 0.0;   // wall time of the last run's iteration loop

static int run_solver(const OMesh &M, const xcal_case &cfg, bool piso, int iterations, i64 ref_cell,
                      double *Uio, double *pio, double *kio, double *wio, double *nutio,
                      double *R_ux, double *R_uy, double *R_uz, double *R_p, int32_t *kry, int32_t *done,
                      double *AUout, double *bUout, double *Apout, double *bpout, std::string &err) {
  i64 nc = M.nc, nf = M.nf;
  int dim = M.dim;
  std::vector<xcal_bc> bcU(cfg.bc_U, cfg.bc_U + cfg.nbc_U), bcp(cfg.bc_p, cfg.bc_p + cfg.nbc_p);
  std::vector<xcal_bc> bck, bcw, bcn;
  bool turb = cfg.model == XCAL_MODEL_KOMEGA;
  if (turb) {
    bck.assign(cfg.bc_k, cfg.bc_k + cfg.nbc_k); bcw.assign(cfg.bc_omega, cfg.bc_omega + cfg.nbc_omega);
    bcn.assign(cfg.bc_nut, cfg.bc_nut + cfg.nbc_nut);
  }
  for (auto *L : {&bcU, &bcp, &bck, &bcw, &bcn})
    for (auto &b : *L) if (b.patch < 0 || b.patch >= (int)M.patches.size()) { err = "BC patch out of range"; return XCAL_ERR_ARG; }
  const double nu = cfg.nu;
  Vec U[3] = {Vec(Uio, Uio + nc), Vec(Uio + nc, Uio + 2 * nc), Vec(Uio + 2 * nc, Uio + 3 * nc)};
  Vec p(pio, pio + nc);
  Vec kf, wf, nut;
  Vec kk, ww;
  if (turb) { kk.assign(kio, kio + nc); ww.assign(wio, wio + nc); nut.assign(nutio, nutio + nc); }
  // simple!/piso! set-up: Solvers_1_SIMPLE.jl:3-67
  Vec gp[3] = {Vec(nc, 0.0), Vec(nc, 0.0), Vec(nc, 0.0)};
  Vec mdotf(nf, 0.0), rDf(nf, 1.0), nueff(nf, 0.0), divHv(nc, 0.0);
  int nU = (dim == 3) ? 3 : 2;
  Eqn ueq[3], peq;
  for (int d = 0; d < 3; ++d) { build_pattern(M, ueq[d].A); ueq[d].b.assign(nc, 0.0); }
  build_pattern(M, peq.A); peq.b.assign(nc, 0.0);
  Terms TU[3], TP;
  for (int d = 0; d < 3; ++d) {
    TU[d].has_time = true; TU[d].time = cfg.schemes_U.time; TU[d].dt = cfg.dt;
    TU[d].has_div = true; TU[d].div = cfg.schemes_U.divergence; TU[d].mdot = &mdotf;
    TU[d].has_lap = true; TU[d].lap_sign = -1; TU[d].gamma = &nueff;
    TU[d].nsrc = 1; TU[d].src[0] = &gp[d]; TU[d].src_sign[0] = -1;
    TU[d].phi = &U[d];
  }
  TP.has_lap = true; TP.lap_sign = 1; TP.gamma = &rDf; TP.nsrc = 1; TP.src[0] = &divHv; TP.src_sign[0] = 1;
  TP.phi = &p;
  Precon PU, PP;
  {  // set_preconditioner: discretise with prev = ConstantScalar(0) then BCs
    Vec zero(nc, 0.0);
    discretise(M, ueq[0], TU[0], zero); apply_bcs(M, ueq[0], TU[0], bcU, 0);
    PU.setup(cfg.solver_U.preconditioner, &ueq[0].A); PU.update();
    discretise(M, peq, TP, zero); apply_bcs(M, peq, TP, bcp, 0);
    PP.setup(cfg.solver_p.preconditioner, &peq.A); PP.update();
  }
  // k-omega initialise_RANS: RANSModels_kOmega.jl:172-234
  Vec nutf(nf, 0.0), nueffk(nf, 0.0), nueffw(nf, 0.0), Dkf(nc, 0.0), Dwf(nc, 0.0), Pk(nc, 0.0), Pw(nc, 0.0);
  Vec G[9];
  // k_eqn and omega_eqn are built on p_eqn.equation (initialise_RANS, :178-207):
  // one storage for the three systems, as in the reference
  Eqn &keq = peq, &weq = peq;
  Terms TK, TW; Precon PK, PW;
  const double bplus = 0.09, alpha1 = 0.52, beta1c = 0.072, sigk = 0.5, sigw = 0.5;   // get_coeffs :152-160
  if (turb) {
    for (int i = 0; i < 9; ++i) G[i].assign(nc, 0.0);
    TK.has_time = true; TK.time = cfg.schemes_k.time; TK.dt = cfg.dt;
    TK.has_div = true; TK.div = cfg.schemes_k.divergence; TK.mdot = &mdotf;
    TK.has_lap = true; TK.lap_sign = -1; TK.gamma = &nueffk; TK.has_si = true; TK.si = &Dkf;
    TK.nsrc = 1; TK.src[0] = &Pk; TK.src_sign[0] = 1; TK.phi = &kk;
    TW = TK; TW.time = cfg.schemes_omega.time; TW.div = cfg.schemes_omega.divergence;
    TW.gamma = &nueffw; TW.si = &Dwf; TW.src[0] = &Pw; TW.phi = &ww;
    Vec zero(nc, 0.0);
    discretise(M, keq, TK, zero); apply_bcs(M, keq, TK, bck, 0);
    PK.setup(cfg.solver_k.preconditioner, &keq.A); PK.update();
    discretise(M, weq, TW, zero); apply_bcs(M, weq, TW, bcw, 0);
    PW.setup(cfg.solver_omega.preconditioner, &weq.A); PW.update();
  }
  // SIMPLE_loop / PISO_loop: Solvers_1_SIMPLE.jl:69-231, Solvers_2_PISO.jl:69-239
  Vec Uf[3] = {Vec(nf, 0.0), Vec(nf, 0.0), Vec(nf, 0.0)};
  Vec pf(nf, 0.0), Hv[3] = {Vec(nc, 0.0), Vec(nc, 0.0), Vec(nc, 0.0)}, rD(nc, 0.0), prev(nc, 0.0);
  for (int i = 0; i < iterations; ++i) { R_ux[i] = 1.0; R_uy[i] = 1.0; if (R_uz) R_uz[i] = 1.0; R_p[i] = 1.0; }
  if (kry) for (int i = 0; i < 5 * iterations; ++i) kry[i] = 0;
  Vec *Up[3] = {&U[0], &U[1], &U[2]};
  Vec *Hp[3] = {&Hv[0], &Hv[1], &Hv[2]};
  interpolate_v(M, Uf, Up, nU);
  correct_boundaries_v(M, Uf, Up, bcU);
  flux(M, mdotf, Uf);
  grad_scalar(M, cfg.schemes_p.gradient, gp[0], gp[1], gp[2], pf, p, bcp);
  for (i64 f = 0; f < nf; ++f) nueff[f] = turb ? nu + nutf[f] : nu;   // update_nueff!
  const double alphaU = cfg.solver_U.relax, alphap = cfg.solver_p.relax;
  int it_done = 0;
  Vec *Rarr[3] = {nullptr, nullptr, nullptr};
  double *Rout[3] = {R_ux, R_uy, R_uz};
  (void)Rarr;
  const auto t_loop0 = std::chrono::steady_clock::now();   // the loop alone (set-up excluded)
  for (int iteration = 0; iteration < iterations; ++iteration) {
    it_done = iteration + 1;
    for (int d = 0; d < nU; ++d) {
      prev = U[d];
      discretise(M, ueq[d], TU[d], prev);
      apply_bcs(M, ueq[d], TU[d], bcU, d);
      if (!piso) implicit_relaxation(ueq[d], prev, alphaU);
      PU.update();   // uy (and uz) reuse ux's preconditioner object (holds ux's A)
      int it = krylov_solve(cfg.solver_U.solver, ueq[d].A, ueq[d].b, U[d], PU, cfg.solver_U.itmax,
                            cfg.solver_U.atol, cfg.solver_U.rtol, nullptr);
      if (kry) kry[5 * iteration + d] = it;
      double r = residual(ueq[d], U[d]);
      if (Rout[d]) Rout[d][iteration] = r;
    }
    for (i64 c = 0; c < nc; ++c) rD[c] = M.cvol[c] / ueq[0].A.nzval[ueq[0].A.pos(c, c)];   // inverse_diagonal!
    interpolate_s(M, rDf, rD);
    for (int d = 0; d < nU; ++d)   // remove_pressure_source!, source sign -1
      for (i64 c = 0; c < nc; ++c) ueq[d].b[c] -= -1.0 * gp[d][c] * M.cvol[c];
    int ncorr = piso ? 2 : 1;
    for (int corr = 0; corr < ncorr; ++corr) {
      // H!: Solvers_0_functions.jl:110-140 (ux's diagonal for every component)
      for (i64 c = 0; c < nc; ++c) {
        double sum[3] = {0.0, 0.0, 0.0};
        for (i64 k = M.cf_ptr[c]; k < M.cf_ptr[c + 1]; ++k) {
          i64 nID = M.cf_nbr[k];
          for (int d = 0; d < nU; ++d) sum[d] += ueq[d].A.get(c, nID) * U[d][nID];
        }
        double D = ueq[0].A.get(c, c);
        double rDc = 1 / D;
        for (int d = 0; d < nU; ++d) Hv[d][c] = (ueq[d].b[c] - sum[d]) * rDc;
        if (nU == 2) Hv[2][c] = 0.0;
      }
      interpolate_v(M, Uf, Hp, nU);
      correct_boundaries_v(M, Uf, Hp, bcU);
      divergence(M, divHv, Uf);
      prev = p;
      discretise(M, peq, TP, prev);
      apply_bcs(M, peq, TP, bcp, 0);
      set_reference(peq, cfg.has_pref != 0, cfg.pref, ref_cell);
      PP.update();
      int it = krylov_solve(cfg.solver_p.solver, peq.A, peq.b, p, PP, cfg.solver_p.itmax,
                            cfg.solver_p.atol, cfg.solver_p.rtol, nullptr);
      if (kry) kry[5 * iteration + 3] = it;
      explicit_relaxation(p, prev, alphap);
      R_p[iteration] = residual(peq, p);
      grad_scalar(M, cfg.schemes_p.gradient, gp[0], gp[1], gp[2], pf, p, bcp);
      for (i64 c = 0; c < nc; ++c)    // correct_velocity!
        for (int d = 0; d < nU; ++d) U[d][c] = Hv[d][c] - gp[d][c] * rD[c];
      interpolate_v(M, Uf, Up, nU);
      correct_boundaries_v(M, Uf, Up, bcU);
      flux(M, mdotf, Uf);
      if (turb) {
        // grad!(gradU, Uf, U, U.BCs): tensor Orthogonal (Calculate_0_gradient.jl:106-112)
        if (cfg.schemes_U.gradient == XCAL_GRAD_MIDPOINT) {
          // interpolate_midpoint! vector (weight*(x1+x2) quirk) then 2x correct+GG
          for (i64 f = 0; f < nf; ++f) {
            double w = M.fweight[f];
            for (int d = 0; d < 3; ++d) Uf[d][f] = w * (U[d][M.o1[f]] + U[d][M.o2[f]]);
          }
          correct_boundaries_v(M, Uf, Up, bcU);
          for (int i = 0; i < 2; ++i)
            for (int d = 0; d < 3; ++d) {
              correct_interpolation(M, G[3 * d], G[3 * d + 1], G[3 * d + 2], Uf[d], U[d]);
              green_gauss(M, G[3 * d], G[3 * d + 1], G[3 * d + 2], Uf[d]);
            }
        } else {
          interpolate_v(M, Uf, Up, nU);
          correct_boundaries_v(M, Uf, Up, bcU);
          for (int d = 0; d < 3; ++d) green_gauss(M, G[3 * d], G[3 * d + 1], G[3 * d + 2], Uf[d]);
        }
        // G[3*d + j] = d U_d / d x_j  -> SMatrix G[j,k] = dU_k/dx_j (xx,yx,zx,xy,...)
        auto Gm = [&](int j, int k, i64 c) { return G[3 * k + j][c]; };
        // turbulence!: RANSModels_kOmega.jl:236-302
        for (i64 c = 0; c < nc; ++c) {   // magnitude2!(Pk, S, scale_factor=2.0)
          double s = 0.0;
          for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) {
              double Sjk = 0.5 * (Gm(j, k, c) + Gm(k, j, c));
              s += Sjk * Sjk;
            }
          Pk[c] = s * 2.0;
        }
        for (i64 c = 0; c < nc; ++c) Pw[c] = alpha1 * Pk[c];
        for (i64 c = 0; c < nc; ++c) Dwf[c] = beta1c * ww[c];
        for (i64 f = 0; f < nf; ++f) nueffw[f] = nu + sigw * nutf[f];
        for (i64 c = 0; c < nc; ++c) Dkf[c] = bplus * ww[c];
        for (i64 f = 0; f < nf; ++f) nueffk[f] = nu + sigk * nutf[f];
        for (i64 c = 0; c < nc; ++c) Pk[c] = nut[c] * Pk[c];
        for (const xcal_bc &bc : bck) {   // correct_production! / set_production! :450-494
          if (bc.type != XCAL_BC_KWALL) continue;
          const OPatch &P = M.patches[bc.patch];
          double ylam = ylam_of(bc.E, bc.kappa);
          double c25 = std::pow(bc.cmu, 0.25);
          for (size_t i = 0; i < P.cells.size(); ++i) {
            i64 c = P.cells[i], f = P.faces[i];
            double delta = M.fdelta[f];
            V3 nrm = M.fnormal[f];
            double uStar = c25 * std::sqrt(kk[c]);
            double dUdy = uStar / (bc.kappa * delta);
            double yplus = c25 * delta * std::sqrt(kk[c]) / nu;
            double nutw = nut_wall(nu, yplus, bc.kappa, bc.E);
            V3 Ud = v3(U[0][c] - 0.0, U[1][c] - 0.0, U[2][c] - 0.0);
            V3 Up2 = vsub(Ud, vscale(nrm, vdot(Ud, nrm)));
            V3 gr = vdiv(Up2, delta);
            double mag = std::sqrt((gr.x * gr.x + gr.y * gr.y) + gr.z * gr.z);
            if (yplus > ylam) Pk[c] = (nu + nutw) * mag * dUdy;
          }
        }
        // omega equation
        prev = ww;
        discretise(M, weq, TW, prev);
        apply_bcs(M, weq, TW, bcw, 0);
        implicit_relaxation(weq, prev, cfg.solver_omega.relax);
        for (const xcal_bc &bc : bcw) {   // constrain_equation! :346-399
          if (bc.type != XCAL_BC_OMEGAWALL) continue;
          const OPatch &P = M.patches[bc.patch];
          double ylam = ylam_of(bc.E, bc.kappa), c25 = std::pow(bc.cmu, 0.25);
          for (size_t i = 0; i < P.cells.size(); ++i) {
            i64 c = P.cells[i], f = P.faces[i];
            double y = M.fdelta[f];
            double wvis = 6.0 * nu / (bc.beta1 * (y * y));
            double wlog = std::sqrt(kk[c]) / (c25 * bc.kappa * y);
            double yplus = c25 * y * std::sqrt(kk[c]) / nu;
            double wc = (yplus > ylam) ? wlog : wvis;
            i64 d = weq.A.pos(c, c);
            weq.b[c] += weq.A.nzval[d] * wc;
            weq.A.nzval[d] += weq.A.nzval[d];
          }
        }
        PW.update();
        krylov_solve(cfg.solver_omega.solver, weq.A, weq.b, ww, PW, cfg.solver_omega.itmax,
                     cfg.solver_omega.atol, cfg.solver_omega.rtol, nullptr);
        for (const xcal_bc &bc : bcw) {   // constrain_boundary! / set_cell_value! :401-448
          if (bc.type != XCAL_BC_OMEGAWALL) continue;
          const OPatch &P = M.patches[bc.patch];
          double ylam = ylam_of(bc.E, bc.kappa), c25 = std::pow(bc.cmu, 0.25);
          for (size_t i = 0; i < P.cells.size(); ++i) {
            i64 c = P.cells[i], f = P.faces[i];
            double y = M.fdelta[f];
            double wvis = 6.0 * nu / (bc.beta1 * (y * y));
            double wlog = std::sqrt(kk[c]) / (c25 * bc.kappa * y);
            double yplus = c25 * y * std::sqrt(kk[c]) / nu;
            ww[c] = (yplus > ylam) ? wlog : wvis;
          }
        }
        bound_field(M, ww, std::numeric_limits<double>::epsilon());
        // k equation
        prev = kk;
        discretise(M, keq, TK, prev);
        apply_bcs(M, keq, TK, bck, 0);
        implicit_relaxation(keq, prev, cfg.solver_k.relax);
        PK.update();
        krylov_solve(cfg.solver_k.solver, keq.A, keq.b, kk, PK, cfg.solver_k.itmax,
                     cfg.solver_k.atol, cfg.solver_k.rtol, nullptr);
        bound_field(M, kk, std::numeric_limits<double>::epsilon());
        for (i64 c = 0; c < nc; ++c) nut[c] = kk[c] / ww[c];   // update_eddy_viscosity!
        interpolate_s(M, nutf, nut);
        correct_boundaries_s(M, nutf, nut, bcn);
        for (const xcal_bc &bc : bcn) {   // correct_eddy_viscosity! / correct_nut_wall! :496-536
          if (bc.type != XCAL_BC_NUTWALL) continue;
          const OPatch &P = M.patches[bc.patch];
          double ylam = ylam_of(bc.E, bc.kappa), c25 = std::pow(bc.cmu, 0.25);
          for (size_t i = 0; i < P.cells.size(); ++i) {
            i64 c = P.cells[i], f = P.faces[i];
            double yplus = c25 * M.fdelta[f] * std::sqrt(kk[c]) / nu;
            double nutw = nut_wall(nu, yplus, bc.kappa, bc.E);
            if (yplus > ylam) nutf[f] = nutw;
          }
        }
        for (i64 f = 0; f < nf; ++f) nueff[f] = nu + nutf[f];   // update_nueff!
      }
    }
    if (!piso) {
      const double convergence = 1e-7;
      bool conv = R_ux[iteration] <= convergence && R_uy[iteration] <= convergence &&
                  R_p[iteration] <= convergence;
      if (dim == 3 && R_uz) conv = conv && R_uz[iteration] <= convergence;
      if (conv) break;
    }
  }
  g_last_loop_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_loop0).count();
  if (done) *done = it_done;
  for (int d = 0; d < 3; ++d) std::copy(U[d].begin(), U[d].end(), Uio + d * nc);
  std::copy(p.begin(), p.end(), pio);
  if (turb) {
    std::copy(kk.begin(), kk.end(), kio); std::copy(ww.begin(), ww.end(), wio);
    std::copy(nut.begin(), nut.end(), nutio);
  }
  // last assembled systems in CSR (row) order
  auto csr_vals = [&](const CSC &A, double *out) {
    i64 k = 0;
    for (i64 r = 0; r < nc; ++r)
      for (i64 q = A.colptr[r]; q < A.colptr[r + 1]; ++q) out[k++] = A.get(r, A.rowval[q]);
  };
  if (AUout) csr_vals(ueq[0].A, AUout);
  if (bUout) for (int d = 0; d < 3; ++d) std::copy(ueq[d].b.begin(), ueq[d].b.end(), bUout + d * nc);
  if (Apout) csr_vals(peq.A, Apout);
  if (bpout) std::copy(peq.b.begin(), peq.b.end(), bpout);
  return XCAL_OK;
}

// ----------------------------------------------------- level sets, renumbering
// DILU level sets of a CSR pattern: forward level = 1 + max level of lower
// neighbours; backward level = 1 + max backward level of upper neighbours.
static void levels_of(i64 n, const int32_t *rp, const int32_t *col, int32_t *fl, int32_t *bl) {
  for (i64 i = 0; i < n; ++i) {
    int32_t l = 0;
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k) if (col[k] < i) l = std::max(l, fl[col[k]] + 1);
    fl[i] = l;
  }
  for (i64 i = n - 1; i >= 0; --i) {
    int32_t l = 0;
    for (int32_t k = rp[i]; k < rp[i + 1]; ++k) if (col[k] > i) l = std::max(l, bl[col[k]] + 1);
    bl[i] = l;
  }
}

// Reverse Cuthill-McKee on the cell adjacency: start at the lowest-degree cell
// (lowest index on ties), BFS visiting neighbours by ascending (degree, index);
// every further component from its own lowest-degree unvisited cell; reverse.
static void rcm_order(i64 n, const std::vector<std::vector<i64>> &adj, std::vector<i64> &perm) {
  std::vector<i64> order; order.reserve(n);
  std::vector<char> vis(n, 0);
  std::vector<i64> deg(n);
  for (i64 i = 0; i < n; ++i) deg[i] = (i64)adj[i].size();
  while ((i64)order.size() < n) {
    i64 s = -1;
    for (i64 i = 0; i < n; ++i) if (!vis[i] && (s < 0 || deg[i] < deg[s])) s = i;
    size_t head = order.size();
    order.push_back(s); vis[s] = 1;
    while (head < order.size()) {
      i64 u = order[head++];
      std::vector<i64> nb;
      for (i64 v : adj[u]) if (!vis[v]) { nb.push_back(v); vis[v] = 1; }
      std::sort(nb.begin(), nb.end(), [&](i64 a, i64 b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; });
      for (i64 v : nb) order.push_back(v);
    }
  }
  perm.assign(n, 0);
  for (i64 k = 0; k < n; ++k) perm[order[n - 1 - k]] = k;
}
// Multicolour classes: two colours by BFS when the adjacency is bipartite,
// otherwise greedy smallest-colour in index order.  New numbering: colour by
// colour, original order inside a colour.
static void color_order(i64 n, const std::vector<std::vector<i64>> &adj, std::vector<i64> &perm) {
  std::vector<int> color(n, -1);
  bool bip = true;
  for (i64 s = 0; s < n && bip; ++s) {
    if (color[s] >= 0) continue;
    color[s] = 0;
    std::vector<i64> q{s};
    for (size_t h = 0; h < q.size() && bip; ++h) {
      i64 u = q[h];
      for (i64 v : adj[u]) {
        if (color[v] < 0) { color[v] = 1 - color[u]; q.push_back(v); }
        else if (color[v] == color[u]) { bip = false; break; }
      }
    }
  }
  if (!bip) {
    std::fill(color.begin(), color.end(), -1);
    for (i64 i = 0; i < n; ++i) {
      std::vector<char> used(adj[i].size() + 2, 0);
      for (i64 v : adj[i]) if (color[v] >= 0 && color[v] < (int)used.size()) used[color[v]] = 1;
      int c = 0;
      while (used[c]) c++;
      color[i] = c;
    }
  }
  int nc = 0;
  for (i64 i = 0; i < n; ++i) nc = std::max(nc, color[i] + 1);
  perm.assign(n, 0);
  i64 k = 0;
  for (int c = 0; c < nc; ++c)
    for (i64 i = 0; i < n; ++i) if (color[i] == c) perm[i] = k++;
}

// ================================================================ C API
struct orc_mesh_s { OMesh M; };
typedef orc_mesh_s *orc_mesh;

extern "C" {

int orc_build_unv(const char *path, double scale, orc_mesh *out, char *err, size_t nerr) {
  auto *h = new orc_mesh_s();
  std::string e;
  int st = build_mesh_unv(path, scale, h->M, e);
  if (st) { if (err && nerr) snprintf(err, nerr, "%s", e.c_str()); delete h; return st; }
  mesh_export_prepare(h->M);
  *out = h;
  return XCAL_OK;
}

int orc_mesh_from_desc(const xcal_mesh_desc *d, orc_mesh *out, char *err, size_t nerr) {
  auto *h = new orc_mesh_s();
  std::string e;
  int st = mesh_from_desc(d, h->M, e);
  if (st) { if (err && nerr) snprintf(err, nerr, "%s", e.c_str()); delete h; return st; }
  mesh_export_prepare(h->M);
  *out = h;
  return XCAL_OK;
}

void orc_mesh_free(orc_mesh m) { delete m; }

int orc_mesh_counts(orc_mesh m, int64_t *c) {
  const OMesh &M = m->M;
  c[0] = M.nc; c[1] = M.nf; c[2] = M.nbf; c[3] = M.cf_ptr[M.nc]; c[4] = (i64)M.patches.size();
  c[5] = (i64)M.x_pf.size(); c[6] = M.nnodes; c[7] = (i64)M.names.size();
  return XCAL_OK;
}

int orc_mesh_desc(orc_mesh m, xcal_mesh_desc *d) {
  OMesh &M = m->M;
  d->ncells = M.nc; d->nfaces = M.nf; d->nbfaces = M.nbf; d->dim = M.dim;
  d->cell_centre = M.x_cc.data(); d->cell_volume = M.cvol.data();
  d->cell_faces_ptr = M.x_cfp.data(); d->cell_faces = M.x_cf.data();
  d->cell_neighbours = M.x_cn.data(); d->cell_nsign = M.x_cs.data();
  d->face_owner = M.x_own.data(); d->face_centre = M.x_fc.data(); d->face_normal = M.x_fn.data();
  d->face_e = M.x_fe.data(); d->face_area = M.farea.data(); d->face_delta = M.fdelta.data();
  d->face_weight = M.fweight.data(); d->npatches = (i64)M.patches.size();
  d->patch_ptr = M.x_pptr.data(); d->patch_faces = M.x_pf.data(); d->patch_cells = M.x_pc.data();
  return XCAL_OK;
}

int orc_mesh_patch_names(orc_mesh m, char *buf, size_t n) {
  snprintf(buf, n, "%s", m->M.names.c_str());
  return XCAL_OK;
}

// CSC pattern of Equation(mesh) (0-based colptr/rowval)
int orc_mesh_pattern(orc_mesh m, int64_t *colptr, int64_t *rowval) {
  CSC A;
  build_pattern(m->M, A);
  for (i64 i = 0; i <= A.n; ++i) colptr[i] = A.colptr[i];
  for (size_t k = 0; k < A.rowval.size(); ++k) rowval[k] = A.rowval[k];
  return XCAL_OK;
}

int orc_run(orc_mesh m, const xcal_case *cfg, int32_t piso, int32_t iterations, int64_t ref_cell,
            double *U, double *p, double *k, double *w, double *nut, double *R_ux, double *R_uy,
            double *R_uz, double *R_p, int32_t *kry, int32_t *done, double *AU, double *bU,
            double *Ap, double *bp, char *err, size_t nerr) {
  std::string e;
  int st = run_solver(m->M, *cfg, piso != 0, iterations, ref_cell, U, p, k, w, nut, R_ux, R_uy, R_uz,
                      R_p, kry, done, AU, bU, Ap, bp, e);
  if (st && err && nerr) snprintf(err, nerr, "%s", e.c_str());
  return st;
}

// discretise! (+ apply_boundary_conditions! when nbc > 0) of a user-built model
// equation on the mesh: vals in CSR (row) order of the mesh's pattern (the
// pattern arrays of orc_mesh_pattern read as row_ptr/col), b per cell.  comp
// selects the component of vector BC values.
int orc_assemble(orc_mesh m, const xcal_term *terms, int32_t nterms, const xcal_source *srcs, int32_t nsrc,
                 const xcal_bc *bcs, int32_t nbc, int32_t comp, const double *phi, const double *prev, double dt,
                 double *vals, double *b) {
  const OMesh &M = m->M;
  for (int q = 0; q < nbc; ++q)
    if (bcs[q].patch < 0 || bcs[q].patch >= (int)M.patches.size()) return XCAL_ERR_ARG;
  Eqn E;
  build_pattern(M, E.A);
  E.b.assign(M.nc, 0.0);
  discretise_terms(M, E, terms, nterms, srcs, nsrc, prev, dt);
  if (nbc > 0) apply_bcs_terms(M, E, terms, nterms, bcs, nbc, phi, comp);
  i64 k = 0;   // CSR (row) order of the pattern
  for (i64 r = 0; r < M.nc; ++r)
    for (i64 q = E.A.colptr[r]; q < E.A.colptr[r + 1]; ++q) vals[k++] = E.A.get(r, E.A.rowval[q]);
  std::copy(E.b.begin(), E.b.end(), b);
  return XCAL_OK;
}

// CSC of A from its CSR arrays (row_ptr/col 0-based, columns ascending).
static CSC csc_of_csr(int64_t n, const int32_t *rp, const int32_t *col, const double *val) {
  CSC A;
  A.n = n;
  A.colptr.assign(n + 1, 0);
  for (i64 i = 0; i < n; ++i) for (int32_t q = rp[i]; q < rp[i + 1]; ++q) A.colptr[col[q] + 1]++;
  for (i64 j = 0; j < n; ++j) A.colptr[j + 1] += A.colptr[j];
  A.rowval.assign(A.colptr[n], 0);
  A.nzval.assign(A.colptr[n], 0.0);
  std::vector<i64> fill(A.colptr.begin(), A.colptr.end() - 1);
  for (i64 i = 0; i < n; ++i)
    for (int32_t q = rp[i]; q < rp[i + 1]; ++q) {
      const i64 pos = fill[col[q]]++;
      A.rowval[pos] = i;
      A.nzval[pos] = val[q];
    }
  return A;
}

// mul!(y, A, x) (CSC column scatter, Solvers_0_functions.jl:18) of a CSR matrix.
int orc_csr_spmv(int64_t n, const int32_t *rp, const int32_t *col, const double *val, const double *x, double *y) {
  CSC A = csc_of_csr(n, rp, col, val);
  std::vector<double> xx(x, x + n), yy(n);
  spmv(A, xx, yy);
  std::copy(yy.begin(), yy.end(), y);
  return XCAL_OK;
}

// grad!(grad_phi) Orthogonal of a scalar cell field with the given conditions
// (Calculate_0_gradient.jl:96-112): grad as x, y, z arrays of ncells each.
int orc_grad(orc_mesh m, const double *phi, const xcal_bc *bcs, int32_t nbc, double *grad) {
  const OMesh &M = m->M;
  for (int q = 0; q < nbc; ++q)
    if (bcs[q].patch < 0 || bcs[q].patch >= (int)M.patches.size()) return XCAL_ERR_ARG;
  std::vector<xcal_bc> bc(bcs, bcs + nbc);
  Vec p(phi, phi + M.nc), dx(M.nc), dy(M.nc), dz(M.nc), pf(M.nf);
  grad_scalar(M, XCAL_GRAD_ORTHOGONAL, dx, dy, dz, pf, p, bc);
  std::copy(dx.begin(), dx.end(), grad);
  std::copy(dy.begin(), dy.end(), grad + M.nc);
  std::copy(dz.begin(), dz.end(), grad + 2 * M.nc);
  return XCAL_OK;
}

// Seconds spent in the iteration loop of the last orc_run (its set-up excluded).
double orc_last_loop_seconds() { return g_last_loop_seconds; }

// run!(eqn) on a CSR matrix (pattern symmetric, columns sorted).
int orc_linear_solve(int32_t solver, int32_t precon, int64_t n, const int32_t *rp, const int32_t *col,
                     const double *val, const double *b, double *x, int32_t itmax, double atol,
                     double rtol, int32_t *niter, double *rnorm) {
  // CSR of A is the CSC of A^T; build the CSC of A itself
  CSC A; A.n = n; A.colptr.assign(n + 1, 0);
  for (i64 i = 0; i < n; ++i) for (int32_t q = rp[i]; q < rp[i + 1]; ++q) A.colptr[col[q] + 1]++;
  for (i64 j = 0; j < n; ++j) A.colptr[j + 1] += A.colptr[j];
  A.rowval.assign(A.colptr[n], 0); A.nzval.assign(A.colptr[n], 0.0);
  std::vector<i64> fill(A.colptr.begin(), A.colptr.end() - 1);
  for (i64 i = 0; i < n; ++i)
    for (int32_t q = rp[i]; q < rp[i + 1]; ++q) {
      i64 j = col[q], pos = fill[j]++;
      A.rowval[pos] = i; A.nzval[pos] = val[q];
    }
  Precon M; M.setup(precon, &A); M.update();
  std::vector<double> bb(b, b + n), xx(x, x + n);
  double rn = 0.0;
  int it = krylov_solve(solver, A, bb, xx, M, itmax, atol, rtol, &rn);
  std::copy(xx.begin(), xx.end(), x);
  if (niter) *niter = it;
  if (rnorm) *rnorm = rn;
  return XCAL_OK;
}

// Any preconditioner applied once (update_preconditioner! + ldiv!), CSR input.
int orc_precon_apply(int32_t precon, int64_t n, const int32_t *rp, const int32_t *col, const double *val,
                     const double *b, double *y) {
  CSC A; A.n = n; A.colptr.assign(n + 1, 0);
  for (i64 i = 0; i < n; ++i) for (int32_t q = rp[i]; q < rp[i + 1]; ++q) A.colptr[col[q] + 1]++;
  for (i64 j = 0; j < n; ++j) A.colptr[j + 1] += A.colptr[j];
  A.rowval.assign(A.colptr[n], 0); A.nzval.assign(A.colptr[n], 0.0);
  std::vector<i64> fill(A.colptr.begin(), A.colptr.end() - 1);
  for (i64 i = 0; i < n; ++i)
    for (int32_t q = rp[i]; q < rp[i + 1]; ++q) {
      i64 j = col[q], pos = fill[j]++;
      A.rowval[pos] = i; A.nzval[pos] = val[q];
    }
  Precon M; M.setup(precon, &A); M.update();
  std::vector<double> bb(b, b + n), yy(n, 0.0);
  M.apply(bb, yy);
  std::copy(yy.begin(), yy.end(), y);
  return XCAL_OK;
}

// DILU preconditioner applied once (update + ldiv!) -- for unit parity.
int orc_dilu_apply(int64_t n, const int32_t *rp, const int32_t *col, const double *val,
                   const double *b, double *y, double *dinv) {
  CSC A; A.n = n; A.colptr.assign(n + 1, 0);
  for (i64 i = 0; i < n; ++i) for (int32_t q = rp[i]; q < rp[i + 1]; ++q) A.colptr[col[q] + 1]++;
  for (i64 j = 0; j < n; ++j) A.colptr[j + 1] += A.colptr[j];
  A.rowval.assign(A.colptr[n], 0); A.nzval.assign(A.colptr[n], 0.0);
  std::vector<i64> fill(A.colptr.begin(), A.colptr.end() - 1);
  for (i64 i = 0; i < n; ++i)
    for (int32_t q = rp[i]; q < rp[i + 1]; ++q) {
      i64 j = col[q], pos = fill[j]++;
      A.rowval[pos] = i; A.nzval[pos] = val[q];
    }
  Precon M; M.setup(XCAL_PRECON_DILU, &A); M.update();
  std::vector<double> bb(b, b + n), yy(n);
  M.apply(bb, yy);
  std::copy(yy.begin(), yy.end(), y);
  if (dinv) std::copy(M.D.begin(), M.D.end(), dinv);
  return XCAL_OK;
}

// residual!(R, equation, phi) on a CSR system (Solvers_0_functions.jl:13-63)
double orc_residual(int64_t n, const int32_t *rp, const int32_t *col, const double *val, const double *x,
                    const double *b) {
  Eqn E;
  E.A.n = n; E.A.colptr.assign(n + 1, 0);
  for (i64 i = 0; i < n; ++i) for (int32_t q = rp[i]; q < rp[i + 1]; ++q) E.A.colptr[col[q] + 1]++;
  for (i64 j = 0; j < n; ++j) E.A.colptr[j + 1] += E.A.colptr[j];
  E.A.rowval.assign(E.A.colptr[n], 0); E.A.nzval.assign(E.A.colptr[n], 0.0);
  std::vector<i64> fill(E.A.colptr.begin(), E.A.colptr.end() - 1);
  for (i64 i = 0; i < n; ++i)
    for (int32_t q = rp[i]; q < rp[i + 1]; ++q) {
      i64 j = col[q], pos = fill[j]++;
      E.A.rowval[pos] = i; E.A.nzval[pos] = val[q];
    }
  E.b.assign(b, b + n);
  std::vector<double> xx(x, x + n);
  return residual(E, xx);
}

double orc_canon_dot(int64_t n, const double *x, const double *y) {
  return canon_sum_f(n, [&](i64 i) { return x[i] * y[i]; });
}

int orc_levels(int64_t n, const int32_t *rp, const int32_t *col, int32_t *fl, int32_t *bl) {
  levels_of(n, rp, col, fl, bl);
  return XCAL_OK;
}

// Cell renumbering (mode 1 RCM, 2 colour) of a mesh's adjacency; perm[old] = new (0-based).
int orc_renumber(orc_mesh m, int32_t mode, int64_t *perm) {
  const OMesh &M = m->M;
  std::vector<std::vector<i64>> adj(M.nc);
  for (i64 c = 0; c < M.nc; ++c) {
    for (i64 k = M.cf_ptr[c]; k < M.cf_ptr[c + 1]; ++k) adj[c].push_back(M.cf_nbr[k]);
    std::sort(adj[c].begin(), adj[c].end());
    adj[c].erase(std::unique(adj[c].begin(), adj[c].end()), adj[c].end());
  }
  std::vector<i64> pm;
  if (mode == XCAL_RENUMBER_RCM) rcm_order(M.nc, adj, pm);
  else if (mode == XCAL_RENUMBER_COLOR) color_order(M.nc, adj, pm);
  else { pm.resize(M.nc); for (i64 i = 0; i < M.nc; ++i) pm[i] = i; }
  std::copy(pm.begin(), pm.end(), perm);
  return XCAL_OK;
}

}  // extern "C"
