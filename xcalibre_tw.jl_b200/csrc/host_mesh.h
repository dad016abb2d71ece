// Host-side mesh construction and device-layout preparation for libxcal.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/xcal.h"

namespace xcal {

// Reference-layout mesh held on the host, 0-based.
struct HostMesh {
  int64_t nc = 0, nf = 0, nbf = 0, nnodes = 0;
  int dim = 2;
  std::vector<double> cc, cvol;                      // cc [3*nc]
  std::vector<int64_t> cf_ptr, cf_face, cf_nbr, cf_sign;
  std::vector<int64_t> o1, o2;
  std::vector<double> fc, fn, fe, farea, fdelta, fweight;   // fc/fn/fe [3*nf]
  std::vector<std::string> pname;
  std::vector<int64_t> pptr, pfaces, pcells;       // concatenated patches
  std::vector<double> nodes;                       // [3*nnodes] (optional: VTK output)
  std::vector<int64_t> cn_ptr, cn;                 // cell node lists, 0-based (optional)
  // 1-based export copies (xcal_hmesh_desc)
  std::vector<int64_t> x_cfp, x_cf, x_cn, x_own, x_pf, x_pc, x_cnp, x_cnode;
  std::string names;
  void prepare_export();
};

int build_unv(const char *path, double scale, HostMesh &M, std::string &err);
int mesh_from_desc(const xcal_mesh_desc *d, HostMesh &M, std::string &err);

// Cell renumbering: perm[old] = new.
void renumber_perm(const HostMesh &M, int mode, std::vector<int64_t> &perm);
// Apply a permutation (cells) and, for a non-identity mode, sort internal faces
// by (min owner, max owner, old id); per-cell face lists re-sorted by face id.
void apply_perm(const HostMesh &in, const std::vector<int64_t> &perm, bool reorder_faces,
                HostMesh &out);

// Device-ready integer structures built from a (renumbered) mesh.  Matrix and
// per-cell face lists use an ELL layout padded to np = 256*ceil(n/256) rows:
// entry k of row i sits at k*np + i (coalesced across a warp); unused entries
// hold column -1.  Entries of a row are in ascending column order.
struct Prep {
  int n = 0, nf = 0, nbf = 0, nnz = 0, np = 0, W = 0, Wf = 0;
  std::vector<int> row_ptr, col, diag, tslot;   // CSR view (export, tests)
  std::vector<int> e_col, e_tpos, dpos, csr2ell;
  std::vector<int> f_face, f_nbr, f_pos;
  std::vector<signed char> f_sign;
  std::vector<unsigned char> f_first;
  std::vector<int> cb_ptr, cb_face;          // boundary faces per cell, face-id order
  std::vector<int> flev, blev;
  int nfl = 0, nbl = 0;
  std::vector<int> o1, o2;
};
int prepare(const HostMesh &M, Prep &P, std::string &err);

}  // namespace xcal
