// Host mesh builder and device-layout preparation.
//
// build_unv() produces the reference's flattened mesh from a UNV file with the
// same numbering rules as build_mesh + update_mesh_format
// (src/UNV2/UNV2_1_loader.jl:3-120, src/UNV2/UNV2_3_builder.jl:3-288,
// src/UNV2/UNV2_2_geometry.jl:11-165, src/Mesh/Mesh2D/Mesh2D_0_update_mesh.jl:5-142),
// in O(faces) instead of the reference's O(boundary faces^2) boundary search:
// hash maps replace unique! and the linear face search; geometry uses the same
// floating-point operation order, so results are bitwise equal.
#include "host_mesh.h"

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <numeric>
#include <unordered_map>

namespace xcal {

namespace {

struct P3 { double x, y, z; };
inline P3 add(P3 a, P3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline P3 scl(P3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline P3 dvd(P3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(P3 a, P3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline double nrm(P3 a) { return std::sqrt((a.x * a.x + a.y * a.y) + a.z * a.z); }
inline P3 crs(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }

inline uint64_t key2(int64_t a, int64_t b) { return ((uint64_t)a << 32) ^ (uint64_t)b; }

// whitespace tokeniser over one line (no allocation per token beyond the vector)
inline void split(const std::string &line, std::vector<std::string> &out) {
  out.clear();
  size_t i = 0, n = line.size();
  while (i < n) {
    while (i < n && (line[i] == ' ' || line[i] == '\t' || line[i] == '\r')) i++;
    size_t j = i;
    while (j < n && !(line[j] == ' ' || line[j] == '\t' || line[j] == '\r')) j++;
    if (j > i) out.emplace_back(line, i, j - i);
    i = j;
  }
}
inline bool to_i64(const std::string &s, int64_t &v) {
  if (s.empty()) return false;
  char *end = nullptr;
  errno = 0;
  long long r = strtoll(s.c_str(), &end, 10);
  if (*end || errno) return false;
  v = r;
  return true;
}

}  // namespace

void HostMesh::prepare_export() {
  x_cfp.resize(nc + 1);
  for (int64_t c = 0; c <= nc; ++c) x_cfp[c] = cf_ptr[c] + 1;
  size_t tot = cf_face.size();
  x_cf.resize(tot); x_cn.resize(tot);
  for (size_t k = 0; k < tot; ++k) { x_cf[k] = cf_face[k] + 1; x_cn[k] = cf_nbr[k] + 1; }
  x_own.resize(2 * nf);
  for (int64_t f = 0; f < nf; ++f) { x_own[2 * f] = o1[f] + 1; x_own[2 * f + 1] = o2[f] + 1; }
  x_pf.resize(pfaces.size()); x_pc.resize(pcells.size());
  for (size_t k = 0; k < pfaces.size(); ++k) { x_pf[k] = pfaces[k] + 1; x_pc[k] = pcells[k] + 1; }
  names.clear();
  for (auto &s : pname) { names += s; names += "\n"; }
  x_cnp.clear(); x_cnode.clear();
  if (!cn_ptr.empty()) {
    x_cnp.resize(cn_ptr.size());
    for (size_t c = 0; c < cn_ptr.size(); ++c) x_cnp[c] = cn_ptr[c] + 1;
    x_cnode.resize(cn.size());
    for (size_t k = 0; k < cn.size(); ++k) x_cnode[k] = cn[k] + 1;
  }
}

int build_unv(const char *path, double scale, HostMesh &M, std::string &err) {
  std::ifstream in(path);
  if (!in) { err = std::string("cannot open ") + path; return XCAL_ERR_IO; }
  std::vector<P3> pts;
  struct El { int64_t vc; int64_t v[4]; int nv; };
  std::vector<El> els;
  struct Grp { std::string name; std::vector<int64_t> el; };
  std::vector<Grp> grps;
  bool blk = false, d11 = false, d12 = false, d67 = false;
  int64_t vcount = 0;
  std::string line;
  std::vector<std::string> s;
  while (std::getline(in, line)) {
    split(line, s);
    if (s.empty()) continue;
    if (!blk && s[0] == "-1") { blk = true; continue; }
    if (blk && s[0] == "-1") { blk = d11 = d12 = d67 = false; continue; }
    if (blk && !d11 && !d12 && !d67) {
      if (s[0] == "2411") { d11 = true; continue; }
      if (s[0] == "2412") { d12 = true; continue; }
      if (s[0] == "2467") { d67 = true; continue; }
    }
    if (d11) {
      if (s[0].find('.') != std::string::npos) {
        if (s.size() < 3) { err = "bad node line"; return XCAL_ERR_MESH; }
        pts.push_back({strtod(s[0].c_str(), nullptr), strtod(s[1].c_str(), nullptr),
                       strtod(s[2].c_str(), nullptr)});
        continue;
      }
    }
    if (d12) {
      int64_t first;
      if (!to_i64(s[0], first)) { err = "bad element line"; return XCAL_ERR_MESH; }
      if (first == 0) continue;
      int64_t last = 0;
      bool lok = to_i64(s.back(), last);
      if (s.size() == 6 && lok && (last == 2 || last == 3 || last == 4)) { vcount = last; continue; }
      if (s.size() >= 2 && s.size() <= 4) {
        El e; e.vc = vcount; e.nv = (int)s.size();
        for (int k = 0; k < e.nv; ++k) if (!to_i64(s[k], e.v[k])) { err = "bad vertex id"; return XCAL_ERR_MESH; }
        els.push_back(e);
        continue;
      }
    }
    if (d67) {
      int64_t a, b;
      if (to_i64(s[0], a) && s.size() > 1 && to_i64(s[1], b) && b == 0) { grps.push_back({"default", {}}); continue; }
      if (!to_i64(s[0], a)) {
        if (grps.empty()) { err = "group name before group header"; return XCAL_ERR_MESH; }
        grps.back().name = s[0]; continue;
      }
      if (grps.empty() || s.size() < 2) { err = "bad group entity line"; return XCAL_ERR_MESH; }
      int64_t e1;
      to_i64(s[1], e1); grps.back().el.push_back(e1);
      if (s.size() >= 6) { int64_t e2; to_i64(s[5], e2); grps.back().el.push_back(e2); }
    }
  }
  if (scale != 1.0) for (auto &p : pts) p = scl(p, scale);
  int64_t np = (int64_t)pts.size();
  int64_t first = -1;
  for (size_t i = 0; i < els.size(); ++i) if (els[i].vc > 2) { first = (int64_t)i; break; }
  if (first < 0) { err = "no 2D elements"; return XCAL_ERR_MESH; }
  int64_t nc = (int64_t)els.size() - first;
  // node -> cells (ascending cell id)
  std::vector<int64_t> ncnt(np + 1, 0);
  for (int64_t c = 0; c < nc; ++c) {
    const El &e = els[first + c];
    for (int k = 0; k < e.nv; ++k) {
      if (e.v[k] < 1 || e.v[k] > np) { err = "element references missing node"; return XCAL_ERR_MESH; }
      ncnt[e.v[k]]++;
    }
  }
  std::vector<int64_t> nptr(np + 2, 0);
  for (int64_t i = 1; i <= np; ++i) nptr[i + 1] = nptr[i] + ncnt[i];
  std::vector<int64_t> ncell(nptr[np + 1]);
  {
    std::vector<int64_t> fill(nptr.begin(), nptr.end());
    for (int64_t c = 0; c < nc; ++c) {
      const El &e = els[first + c];
      for (int k = 0; k < e.nv; ++k) ncell[fill[e.v[k]]++] = c;
    }
  }
  // faces: boundary elements first, then cell edges, first occurrence kept
  std::unordered_map<uint64_t, int64_t> fid;
  fid.reserve((size_t)(nc * 2.2) + 16);
  std::vector<int64_t> fa, fb;
  auto push_face = [&](int64_t a, int64_t b) -> bool {
    if (a == b) return false;
    if (a > b) std::swap(a, b);
    uint64_t k = key2(a, b);
    if (fid.find(k) == fid.end()) { fid.emplace(k, (int64_t)fa.size()); fa.push_back(a); fb.push_back(b); }
    return true;
  };
  int64_t bfaces = 0;
  for (auto &g : grps)
    for (int64_t ei : g.el) {
      if (ei < 1 || ei > (int64_t)els.size() || els[ei - 1].nv < 2) { err = "boundary element out of range"; return XCAL_ERR_MESH; }
      if (!push_face(els[ei - 1].v[0], els[ei - 1].v[1])) { err = "Boundary elements are inconsistent: possible mesh corruption"; return XCAL_ERR_MESH; }
      bfaces++;
    }
  for (int64_t c = 0; c < nc; ++c) {
    const El &e = els[first + c];
    for (int k = 0; k < e.nv; ++k)
      if (!push_face(e.v[k], e.v[(k + 1) % e.nv])) { err = "Boundary elements are inconsistent: possible mesh corruption"; return XCAL_ERR_MESH; }
  }
  int64_t nf = (int64_t)fa.size();
  // face -> owner cells: intersection of the two nodes' cell lists
  std::vector<int64_t> o1(nf), o2(nf);
  std::vector<int64_t> ccount(nc, 0);
  for (int64_t f = 0; f < nf; ++f) {
    int64_t own[2] = {-1, -1};
    int cnt = 0;
    for (int64_t p = nptr[fa[f]]; p < nptr[fa[f] + 1]; ++p)
      for (int64_t q = nptr[fb[f]]; q < nptr[fb[f] + 1]; ++q)
        if (ncell[p] == ncell[q]) {
          if (cnt >= 2) { err = "face shared by more than two cells"; return XCAL_ERR_MESH; }
          own[cnt++] = ncell[p];
        }
    if (cnt == 0) { err = "face without owner cell"; return XCAL_ERR_MESH; }
    o1[f] = own[0]; o2[f] = (cnt == 2) ? own[1] : own[0];
    if (cnt == 2) { ccount[own[0]]++; ccount[own[1]]++; }
  }
  // per-cell face lists in face-id order
  M.cf_ptr.assign(nc + 1, 0);
  for (int64_t c = 0; c < nc; ++c) M.cf_ptr[c + 1] = M.cf_ptr[c] + ccount[c];
  M.cf_face.assign(M.cf_ptr[nc], 0); M.cf_nbr.assign(M.cf_ptr[nc], 0); M.cf_sign.assign(M.cf_ptr[nc], 0);
  {
    std::vector<int64_t> fill(M.cf_ptr.begin(), M.cf_ptr.end() - 1);
    for (int64_t f = 0; f < nf; ++f) {
      if (o1[f] == o2[f]) continue;
      int64_t a = o1[f], b = o2[f];
      M.cf_face[fill[a]] = f; M.cf_nbr[fill[a]] = b; fill[a]++;
      M.cf_face[fill[b]] = f; M.cf_nbr[fill[b]] = a; fill[b]++;
    }
  }
  // boundary connectivity: each patch element matched to its boundary face
  std::unordered_map<uint64_t, int64_t> bmap;
  bmap.reserve((size_t)bfaces * 2 + 16);
  for (int64_t f = 0; f < bfaces && f < nf; ++f) bmap.emplace(key2(fa[f], fb[f]), f);
  M.pname.clear(); M.pptr.assign(1, 0); M.pfaces.clear(); M.pcells.clear();
  for (auto &g : grps) {
    M.pname.push_back(g.name);
    for (int64_t ei : g.el) {
      int64_t a = els[ei - 1].v[0], b = els[ei - 1].v[1];
      if (a > b) std::swap(a, b);
      auto it = bmap.find(key2(a, b));
      if (it != bmap.end()) { M.pfaces.push_back(it->second); M.pcells.push_back(o1[it->second]); }
    }
    M.pptr.push_back((int64_t)M.pfaces.size());
  }
  int64_t nbf = (int64_t)M.pfaces.size();
  // centres (node average, sum from zero)
  M.cc.assign(3 * nc, 0.0);
  for (int64_t c = 0; c < nc; ++c) {
    const El &e = els[first + c];
    P3 sm = {0.0, 0.0, 0.0};
    for (int k = 0; k < e.nv; ++k) sm = add(sm, pts[e.v[k] - 1]);
    P3 ctr = dvd(sm, (double)e.nv);
    M.cc[3 * c] = ctr.x; M.cc[3 * c + 1] = ctr.y; M.cc[3 * c + 2] = ctr.z;
  }
  M.fc.assign(3 * nf, 0.0); M.fn.assign(3 * nf, 0.0); M.fe.assign(3 * nf, 0.0);
  M.farea.assign(nf, 0.0); M.fdelta.assign(nf, 0.0); M.fweight.assign(nf, 0.0);
  for (int64_t f = 0; f < nf; ++f) {
    P3 sm = add(add(P3{0.0, 0.0, 0.0}, pts[fa[f] - 1]), pts[fb[f] - 1]);
    P3 ctr = dvd(sm, 2.0);
    M.fc[3 * f] = ctr.x; M.fc[3 * f + 1] = ctr.y; M.fc[3 * f + 2] = ctr.z;
  }
  auto C3 = [&](int64_t c) { return P3{M.cc[3 * c], M.cc[3 * c + 1], M.cc[3 * c + 2]}; };
  auto F3 = [&](const std::vector<double> &v, int64_t f) { return P3{v[3 * f], v[3 * f + 1], v[3 * f + 2]}; };
  const P3 kk = {0.0, 0.0, 1.0};
  for (int64_t f = nbf; f < nf; ++f) {   // internal faces
    P3 t = sub(pts[fb[f] - 1], pts[fa[f] - 1]);
    double area = nrm(t);
    P3 c1 = C3(o1[f]), c2 = C3(o2[f]), cf = F3(M.fc, f);
    P3 d1f = sub(cf, c1), df2 = sub(c2, cf), d12 = sub(c2, c1);
    P3 normal = crs(dvd(t, area), kk);
    if (dot(d12, normal) < 0.0) normal = scl(normal, -1.0);
    double delta = nrm(d12);
    P3 e = dvd(d12, delta);
    double w = std::fabs(dot(d1f, normal) / (dot(d1f, normal) + dot(df2, normal)));
    M.farea[f] = area; M.fdelta[f] = delta; M.fweight[f] = w;
    M.fn[3 * f] = normal.x; M.fn[3 * f + 1] = normal.y; M.fn[3 * f + 2] = normal.z;
    M.fe[3 * f] = e.x; M.fe[3 * f + 1] = e.y; M.fe[3 * f + 2] = e.z;
  }
  for (int64_t k = 0; k < nbf; ++k) {   // boundary faces, patch order
    int64_t f = M.pfaces[k];
    P3 t = sub(pts[fb[f] - 1], pts[fa[f] - 1]);
    double area = nrm(t);
    P3 normal = crs(dvd(t, area), kk);
    P3 dcf = sub(F3(M.fc, f), C3(o1[f]));
    if (dot(dcf, normal) < 0.0) normal = scl(normal, -1.0);
    double delta = nrm(dcf);
    P3 e = dvd(dcf, delta);
    M.farea[f] = area; M.fdelta[f] = delta; M.fweight[f] = 1.0;
    M.fn[3 * f] = normal.x; M.fn[3 * f + 1] = normal.y; M.fn[3 * f + 2] = normal.z;
    M.fe[3 * f] = e.x; M.fe[3 * f + 1] = e.y; M.fe[3 * f + 2] = e.z;
  }
  M.cvol.assign(nc, 0.0);
  for (int64_t c = 0; c < nc; ++c) {   // nsign and volume
    double vol = 0.0;
    P3 ctr = C3(c);
    for (int64_t k = M.cf_ptr[c]; k < M.cf_ptr[c + 1]; ++k) {
      int64_t f = M.cf_face[k];
      P3 dcf = sub(F3(M.fc, f), ctr);
      P3 n = F3(M.fn, f);
      int64_t s = (dot(dcf, n) > 0.0) ? 1 : -1;
      M.cf_sign[k] = s;
      vol += (dot(dcf, n) * (double)s) * M.farea[f];
    }
    M.cvol[c] = (M.cf_ptr[c + 1] > M.cf_ptr[c]) ? 0.5 * vol : 0.0;
  }
  for (int64_t k = 0; k < nbf; ++k) {
    int64_t f = M.pfaces[k], c = M.pcells[k];
    P3 dcf = sub(F3(M.fc, f), C3(c));
    M.cvol[c] = M.cvol[c] + (0.5 * dot(dcf, F3(M.fn, f))) * M.farea[f];
  }
  M.nc = nc; M.nf = nf; M.nbf = nbf; M.dim = 2; M.nnodes = np;
  M.o1 = o1; M.o2 = o2;
  // mesh.nodes and mesh.cell_nodes (element vertex order), for VTK output
  M.nodes.resize(3 * (size_t)np);
  for (int64_t i = 0; i < np; ++i) { M.nodes[3 * i] = pts[i].x; M.nodes[3 * i + 1] = pts[i].y; M.nodes[3 * i + 2] = pts[i].z; }
  M.cn_ptr.assign(nc + 1, 0);
  M.cn.clear();
  for (int64_t c = 0; c < nc; ++c) {
    const El &e = els[first + c];
    for (int k = 0; k < e.nv; ++k) M.cn.push_back(e.v[k] - 1);
    M.cn_ptr[c + 1] = (int64_t)M.cn.size();
  }
  M.prepare_export();
  return XCAL_OK;
}

int mesh_from_desc(const xcal_mesh_desc *d, HostMesh &M, std::string &err) {
  if (!d || d->ncells <= 0 || d->nfaces <= 0 || d->nbfaces < 0 || d->nbfaces > d->nfaces ||
      d->npatches < 0 || (d->dim != 2 && d->dim != 3)) {
    err = "bad mesh counts or dim"; return XCAL_ERR_ARG;
  }
  if (d->ncells > (int64_t)1 << 30 || d->nfaces > (int64_t)1 << 30) { err = "mesh too large for int32 indices"; return XCAL_ERR_ARG; }
  if (!d->cell_centre || !d->cell_volume || !d->cell_faces_ptr || !d->face_owner || !d->face_area ||
      !d->face_delta || !d->face_weight || !d->face_normal || !d->face_centre || !d->face_e ||
      (d->npatches > 0 && (!d->patch_ptr || !d->patch_faces || !d->patch_cells))) {
    err = "null mesh array"; return XCAL_ERR_ARG;
  }
  int64_t nc = d->ncells, nf = d->nfaces;
  M.nc = nc; M.nf = nf; M.nbf = d->nbfaces; M.dim = d->dim;
  M.cc.assign(d->cell_centre, d->cell_centre + 3 * nc);
  M.cvol.assign(d->cell_volume, d->cell_volume + nc);
  M.cf_ptr.resize(nc + 1);
  for (int64_t c = 0; c <= nc; ++c) M.cf_ptr[c] = d->cell_faces_ptr[c] - 1;
  if (M.cf_ptr[0] != 0) { err = "cell_faces_ptr must start at 1"; return XCAL_ERR_MESH; }
  for (int64_t c = 0; c < nc; ++c) if (M.cf_ptr[c + 1] < M.cf_ptr[c]) { err = "cell_faces_ptr not monotone"; return XCAL_ERR_MESH; }
  int64_t tot = M.cf_ptr[nc];
  if (tot > 0 && (!d->cell_faces || !d->cell_neighbours || !d->cell_nsign)) { err = "null cell face arrays"; return XCAL_ERR_ARG; }
  M.cf_face.resize(tot); M.cf_nbr.resize(tot); M.cf_sign.resize(tot);
  for (int64_t k = 0; k < tot; ++k) {
    M.cf_face[k] = d->cell_faces[k] - 1; M.cf_nbr[k] = d->cell_neighbours[k] - 1; M.cf_sign[k] = d->cell_nsign[k];
    if (M.cf_face[k] < d->nbfaces || M.cf_face[k] >= nf) { err = "cell face id out of range (internal faces only)"; return XCAL_ERR_MESH; }
    if (M.cf_nbr[k] < 0 || M.cf_nbr[k] >= nc) { err = "cell neighbour out of range"; return XCAL_ERR_MESH; }
    if (M.cf_sign[k] != 1 && M.cf_sign[k] != -1) { err = "nsign must be +1 or -1"; return XCAL_ERR_MESH; }
  }
  M.o1.resize(nf); M.o2.resize(nf);
  for (int64_t f = 0; f < nf; ++f) {
    M.o1[f] = d->face_owner[2 * f] - 1; M.o2[f] = d->face_owner[2 * f + 1] - 1;
    if (M.o1[f] < 0 || M.o1[f] >= nc || M.o2[f] < 0 || M.o2[f] >= nc) { err = "face owner out of range"; return XCAL_ERR_MESH; }
  }
  for (int64_t f = 0; f < d->nbfaces; ++f) if (M.o1[f] != M.o2[f]) { err = "faces 1..nbfaces must be boundary faces"; return XCAL_ERR_MESH; }
  for (int64_t c = 0; c < nc; ++c)   // each listed face must join the cell and its neighbour
    for (int64_t k = M.cf_ptr[c]; k < M.cf_ptr[c + 1]; ++k) {
      int64_t f = M.cf_face[k];
      bool ok = (M.o1[f] == c && M.o2[f] == M.cf_nbr[k]) || (M.o2[f] == c && M.o1[f] == M.cf_nbr[k]);
      if (!ok) { err = "cell face list inconsistent with face owners"; return XCAL_ERR_MESH; }
    }
  M.fc.assign(d->face_centre, d->face_centre + 3 * nf);
  M.fn.assign(d->face_normal, d->face_normal + 3 * nf);
  M.fe.assign(d->face_e, d->face_e + 3 * nf);
  M.farea.assign(d->face_area, d->face_area + nf);
  M.fdelta.assign(d->face_delta, d->face_delta + nf);
  M.fweight.assign(d->face_weight, d->face_weight + nf);
  M.pname.clear(); M.pptr.assign(d->npatches + 1, 0); M.pfaces.clear(); M.pcells.clear();
  for (int64_t p = 0; p < d->npatches; ++p) {
    M.pname.push_back("patch" + std::to_string(p));
    if (d->patch_ptr[p + 1] < d->patch_ptr[p]) { err = "patch_ptr not monotone"; return XCAL_ERR_MESH; }
    for (int64_t k = d->patch_ptr[p]; k < d->patch_ptr[p + 1]; ++k) {
      int64_t f = d->patch_faces[k] - 1, c = d->patch_cells[k] - 1;
      if (f < 0 || f >= d->nbfaces || c < 0 || c >= nc || M.o1[f] != c) { err = "patch face/cell inconsistent"; return XCAL_ERR_MESH; }
      M.pfaces.push_back(f); M.pcells.push_back(c);
    }
    M.pptr[p + 1] = (int64_t)M.pfaces.size();
  }
  for (int64_t c = 0; c < nc; ++c) if (!(M.cvol[c] > 0.0)) { err = "non-positive cell volume"; return XCAL_ERR_MESH; }
  M.nodes.clear(); M.cn_ptr.clear(); M.cn.clear(); M.nnodes = 0;
  if (d->nnodes > 0) {
    if (!d->node_coords || !d->cell_nodes_ptr || !d->cell_nodes) { err = "null node arrays"; return XCAL_ERR_ARG; }
    M.nnodes = d->nnodes;
    M.nodes.assign(d->node_coords, d->node_coords + 3 * d->nnodes);
    M.cn_ptr.resize(nc + 1);
    for (int64_t c = 0; c <= nc; ++c) M.cn_ptr[c] = d->cell_nodes_ptr[c] - 1;
    if (M.cn_ptr[0] != 0) { err = "cell_nodes_ptr must start at 1"; return XCAL_ERR_MESH; }
    for (int64_t c = 0; c < nc; ++c) if (M.cn_ptr[c + 1] < M.cn_ptr[c]) { err = "cell_nodes_ptr not monotone"; return XCAL_ERR_MESH; }
    M.cn.resize(M.cn_ptr[nc]);
    for (int64_t k = 0; k < M.cn_ptr[nc]; ++k) {
      M.cn[k] = d->cell_nodes[k] - 1;
      if (M.cn[k] < 0 || M.cn[k] >= d->nnodes) { err = "cell node id out of range"; return XCAL_ERR_MESH; }
    }
  }
  M.prepare_export();
  return XCAL_OK;
}

// ------------------------------------------------------------ renumbering
static void adjacency(const HostMesh &M, std::vector<int64_t> &aptr, std::vector<int64_t> &adj) {
  int64_t n = M.nc;
  aptr.assign(n + 1, 0);
  adj.clear();
  std::vector<int64_t> tmp;
  for (int64_t c = 0; c < n; ++c) {
    tmp.assign(M.cf_nbr.begin() + M.cf_ptr[c], M.cf_nbr.begin() + M.cf_ptr[c + 1]);
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    adj.insert(adj.end(), tmp.begin(), tmp.end());
    aptr[c + 1] = (int64_t)adj.size();
  }
}

void renumber_perm(const HostMesh &M, int mode, std::vector<int64_t> &perm) {
  int64_t n = M.nc;
  perm.resize(n);
  if (mode == XCAL_RENUMBER_NONE) { std::iota(perm.begin(), perm.end(), 0); return; }
  std::vector<int64_t> aptr, adj;
  adjacency(M, aptr, adj);
  if (mode == XCAL_RENUMBER_RCM) {
    // Reverse Cuthill-McKee: each component from its lowest-degree unvisited
    // cell (lowest index on ties); neighbours queued by (degree, index).
    std::vector<int64_t> deg(n), order;
    order.reserve(n);
    for (int64_t i = 0; i < n; ++i) deg[i] = aptr[i + 1] - aptr[i];
    std::vector<int64_t> bydeg(n);
    std::iota(bydeg.begin(), bydeg.end(), 0);
    std::stable_sort(bydeg.begin(), bydeg.end(), [&](int64_t a, int64_t b) { return deg[a] < deg[b]; });
    std::vector<char> vis(n, 0);
    size_t nextstart = 0;
    std::vector<int64_t> nb;
    while ((int64_t)order.size() < n) {
      while (vis[bydeg[nextstart]]) nextstart++;
      int64_t s = bydeg[nextstart];
      size_t head = order.size();
      order.push_back(s); vis[s] = 1;
      while (head < order.size()) {
        int64_t u = order[head++];
        nb.clear();
        for (int64_t k = aptr[u]; k < aptr[u + 1]; ++k) if (!vis[adj[k]]) { nb.push_back(adj[k]); vis[adj[k]] = 1; }
        std::sort(nb.begin(), nb.end(), [&](int64_t a, int64_t b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; });
        order.insert(order.end(), nb.begin(), nb.end());
      }
    }
    for (int64_t k = 0; k < n; ++k) perm[order[n - 1 - k]] = k;
    return;
  }
  // multicolour: BFS two-colouring when bipartite, else greedy smallest colour
  std::vector<int> color(n, -1);
  bool bip = true;
  std::vector<int64_t> q;
  for (int64_t s = 0; s < n && bip; ++s) {
    if (color[s] >= 0) continue;
    color[s] = 0;
    q.assign(1, s);
    for (size_t h = 0; h < q.size() && bip; ++h) {
      int64_t u = q[h];
      for (int64_t k = aptr[u]; k < aptr[u + 1]; ++k) {
        int64_t v = adj[k];
        if (color[v] < 0) { color[v] = 1 - color[u]; q.push_back(v); }
        else if (color[v] == color[u]) { bip = false; break; }
      }
    }
  }
  if (!bip) {
    std::fill(color.begin(), color.end(), -1);
    std::vector<char> used;
    for (int64_t i = 0; i < n; ++i) {
      used.assign(aptr[i + 1] - aptr[i] + 2, 0);
      for (int64_t k = aptr[i]; k < aptr[i + 1]; ++k) {
        int c = color[adj[k]];
        if (c >= 0 && c < (int)used.size()) used[c] = 1;
      }
      int c = 0;
      while (used[c]) c++;
      color[i] = c;
    }
  }
  int ncol = 0;
  for (int64_t i = 0; i < n; ++i) ncol = std::max(ncol, color[i] + 1);
  std::vector<int64_t> cnt(ncol + 1, 0);
  for (int64_t i = 0; i < n; ++i) cnt[color[i] + 1]++;
  for (int c = 0; c < ncol; ++c) cnt[c + 1] += cnt[c];
  for (int64_t i = 0; i < n; ++i) perm[i] = cnt[color[i]]++;
}

void apply_perm(const HostMesh &in, const std::vector<int64_t> &perm, bool reorder_faces, HostMesh &out) {
  int64_t nc = in.nc, nf = in.nf, nbf = in.nbf;
  out = HostMesh();
  out.nc = nc; out.nf = nf; out.nbf = nbf; out.dim = in.dim; out.nnodes = in.nnodes;
  std::vector<int64_t> inv(nc);
  for (int64_t i = 0; i < nc; ++i) inv[perm[i]] = i;
  // face order
  std::vector<int64_t> fperm(nf);   // fperm[old] = new
  std::iota(fperm.begin(), fperm.end(), 0);
  if (reorder_faces && nf > nbf) {
    std::vector<int64_t> ids(nf - nbf);
    std::iota(ids.begin(), ids.end(), nbf);
    auto lo = [&](int64_t f) { return std::min(perm[in.o1[f]], perm[in.o2[f]]); };
    auto hi = [&](int64_t f) { return std::max(perm[in.o1[f]], perm[in.o2[f]]); };
    std::sort(ids.begin(), ids.end(), [&](int64_t a, int64_t b) {
      int64_t la = lo(a), lb = lo(b);
      if (la != lb) return la < lb;
      int64_t ha = hi(a), hb = hi(b);
      if (ha != hb) return ha < hb;
      return a < b;
    });
    for (int64_t k = 0; k < nf - nbf; ++k) fperm[ids[k]] = nbf + k;
  }
  std::vector<int64_t> finv(nf);
  for (int64_t f = 0; f < nf; ++f) finv[fperm[f]] = f;
  out.cc.resize(3 * nc); out.cvol.resize(nc);
  for (int64_t c = 0; c < nc; ++c) {
    int64_t oc = inv[c];
    for (int d = 0; d < 3; ++d) out.cc[3 * c + d] = in.cc[3 * oc + d];
    out.cvol[c] = in.cvol[oc];
  }
  out.nodes = in.nodes;
  if (!in.cn_ptr.empty()) {
    out.cn_ptr.assign(nc + 1, 0);
    for (int64_t c = 0; c < nc; ++c) {
      const int64_t oc = inv[c];
      out.cn.insert(out.cn.end(), in.cn.begin() + in.cn_ptr[oc], in.cn.begin() + in.cn_ptr[oc + 1]);
      out.cn_ptr[c + 1] = (int64_t)out.cn.size();
    }
  }
  out.o1.resize(nf); out.o2.resize(nf);
  out.fc.resize(3 * nf); out.fn.resize(3 * nf); out.fe.resize(3 * nf);
  out.farea.resize(nf); out.fdelta.resize(nf); out.fweight.resize(nf);
  for (int64_t f = 0; f < nf; ++f) {
    int64_t of = finv[f];
    out.o1[f] = perm[in.o1[of]]; out.o2[f] = perm[in.o2[of]];
    for (int d = 0; d < 3; ++d) {
      out.fc[3 * f + d] = in.fc[3 * of + d]; out.fn[3 * f + d] = in.fn[3 * of + d]; out.fe[3 * f + d] = in.fe[3 * of + d];
    }
    out.farea[f] = in.farea[of]; out.fdelta[f] = in.fdelta[of]; out.fweight[f] = in.fweight[of];
  }
  out.cf_ptr.assign(nc + 1, 0);
  for (int64_t c = 0; c < nc; ++c) out.cf_ptr[c + 1] = out.cf_ptr[c] + (in.cf_ptr[inv[c] + 1] - in.cf_ptr[inv[c]]);
  out.cf_face.resize(out.cf_ptr[nc]); out.cf_nbr.resize(out.cf_ptr[nc]); out.cf_sign.resize(out.cf_ptr[nc]);
  std::vector<int64_t> idx;
  for (int64_t c = 0; c < nc; ++c) {
    int64_t oc = inv[c], b = in.cf_ptr[oc], e = in.cf_ptr[oc + 1];
    idx.resize(e - b);
    std::iota(idx.begin(), idx.end(), b);
    std::stable_sort(idx.begin(), idx.end(), [&](int64_t x, int64_t y) { return fperm[in.cf_face[x]] < fperm[in.cf_face[y]]; });
    for (int64_t k = 0; k < e - b; ++k) {
      int64_t src = idx[k], dst = out.cf_ptr[c] + k;
      out.cf_face[dst] = fperm[in.cf_face[src]];
      out.cf_nbr[dst] = perm[in.cf_nbr[src]];
      out.cf_sign[dst] = in.cf_sign[src];
    }
  }
  out.pname = in.pname; out.pptr = in.pptr;
  out.pfaces.resize(in.pfaces.size()); out.pcells.resize(in.pcells.size());
  for (size_t k = 0; k < in.pfaces.size(); ++k) { out.pfaces[k] = fperm[in.pfaces[k]]; out.pcells[k] = perm[in.pcells[k]]; }
  out.prepare_export();
}

// ---------------------------------------------------------- device layout
int prepare(const HostMesh &M, Prep &P, std::string &err) {
  int n = (int)M.nc, nf = (int)M.nf;
  P.n = n; P.nf = nf; P.nbf = (int)M.nbf;
  // CSR pattern: row c = {c} U neighbours(c), ascending, duplicates merged
  P.row_ptr.assign(n + 1, 0);
  P.col.clear();
  std::vector<int> tmp;
  for (int c = 0; c < n; ++c) {
    tmp.clear();
    tmp.push_back(c);
    for (int64_t k = M.cf_ptr[c]; k < M.cf_ptr[c + 1]; ++k) tmp.push_back((int)M.cf_nbr[k]);
    std::sort(tmp.begin(), tmp.end());
    tmp.erase(std::unique(tmp.begin(), tmp.end()), tmp.end());
    P.col.insert(P.col.end(), tmp.begin(), tmp.end());
    P.row_ptr[c + 1] = (int)P.col.size();
  }
  P.nnz = (int)P.col.size();
  auto find = [&](int r, int c) -> int {
    auto b = P.col.begin() + P.row_ptr[r], e = P.col.begin() + P.row_ptr[r + 1];
    auto it = std::lower_bound(b, e, c);
    return (it != e && *it == c) ? (int)(it - P.col.begin()) : -1;
  };
  P.diag.resize(n);
  for (int c = 0; c < n; ++c) P.diag[c] = find(c, c);
  P.tslot.resize(P.nnz);
  for (int r = 0; r < n; ++r)
    for (int k = P.row_ptr[r]; k < P.row_ptr[r + 1]; ++k) {
      P.tslot[k] = find(P.col[k], r);
      if (P.tslot[k] < 0) { err = "matrix pattern not symmetric"; return XCAL_ERR_MESH; }
    }
  // ELL layout of the matrix
  P.np = ((n + 255) / 256) * 256;
  P.W = 0;
  for (int i = 0; i < n; ++i) P.W = std::max(P.W, P.row_ptr[i + 1] - P.row_ptr[i]);
  if (P.W > 64) { err = "more than 63 neighbours in one cell"; return XCAL_ERR_UNSUPPORTED; }
  P.e_col.assign((size_t)P.W * P.np, -1);
  P.e_tpos.assign((size_t)P.W * P.np, -1);
  P.dpos.assign(P.np, 0);
  P.csr2ell.assign(P.nnz, 0);
  for (int i = 0; i < n; ++i)
    for (int k = P.row_ptr[i]; k < P.row_ptr[i + 1]; ++k) {
      int e = (k - P.row_ptr[i]) * P.np + i;
      P.e_col[e] = P.col[k];
      P.csr2ell[k] = e;
    }
  for (int i = 0; i < n; ++i) {
    P.dpos[i] = P.csr2ell[P.diag[i]];
    for (int k = P.row_ptr[i]; k < P.row_ptr[i + 1]; ++k) P.e_tpos[P.csr2ell[k]] = P.csr2ell[P.tslot[k]];
  }
  // cell -> internal face entries (reference order) with their matrix positions
  P.Wf = 0;
  for (int c = 0; c < n; ++c) P.Wf = std::max(P.Wf, (int)(M.cf_ptr[c + 1] - M.cf_ptr[c]));
  P.Wf = std::max(P.Wf, 1);
  P.f_face.assign((size_t)P.Wf * P.np, -1);
  P.f_nbr.assign((size_t)P.Wf * P.np, 0);
  P.f_pos.assign((size_t)P.Wf * P.np, 0);
  P.f_sign.assign((size_t)P.Wf * P.np, 0);
  P.f_first.assign((size_t)P.Wf * P.np, 0);
  for (int c = 0; c < n; ++c) {
    int b = (int)M.cf_ptr[c];
    for (int k = b; k < (int)M.cf_ptr[c + 1]; ++k) {
      int e = (k - b) * P.np + c;
      int nb = (int)M.cf_nbr[k];
      int slot = find(c, nb);
      P.f_face[e] = (int)M.cf_face[k];
      P.f_nbr[e] = nb;
      P.f_pos[e] = P.csr2ell[slot];
      P.f_sign[e] = (signed char)M.cf_sign[k];
      bool first = true;
      for (int q = b; q < k; ++q) if (M.cf_nbr[q] == nb) first = false;
      P.f_first[e] = first ? 1 : 0;
    }
  }
  // boundary faces of each cell in face-id order
  std::vector<int> bc_cnt(n + 1, 0);
  for (int f = 0; f < P.nbf; ++f) bc_cnt[M.o1[f] + 1]++;
  P.cb_ptr.assign(n + 1, 0);
  for (int c = 0; c < n; ++c) P.cb_ptr[c + 1] = P.cb_ptr[c] + bc_cnt[c + 1];
  P.cb_face.resize(P.nbf);
  {
    std::vector<int> fill(P.cb_ptr.begin(), P.cb_ptr.end() - 1);
    for (int f = 0; f < P.nbf; ++f) P.cb_face[fill[M.o1[f]]++] = f;
  }
  // DILU level sets
  P.flev.assign(n, 0); P.blev.assign(n, 0);
  for (int i = 0; i < n; ++i) {
    int l = 0;
    for (int k = P.row_ptr[i]; k < P.diag[i]; ++k) l = std::max(l, P.flev[P.col[k]] + 1);
    P.flev[i] = l;
  }
  for (int i = n - 1; i >= 0; --i) {
    int l = 0;
    for (int k = P.diag[i] + 1; k < P.row_ptr[i + 1]; ++k) l = std::max(l, P.blev[P.col[k]] + 1);
    P.blev[i] = l;
  }
  P.nfl = P.nbl = 1;
  for (int i = 0; i < n; ++i) { P.nfl = std::max(P.nfl, P.flev[i] + 1); P.nbl = std::max(P.nbl, P.blev[i] + 1); }
  P.flev.resize(P.np, 0);
  P.blev.resize(P.np, 0);
  P.o1.resize(nf); P.o2.resize(nf);
  for (int f = 0; f < nf; ++f) { P.o1[f] = (int)M.o1[f]; P.o2[f] = (int)M.o2[f]; }
  return XCAL_OK;
}

}  // namespace xcal
