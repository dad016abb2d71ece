// Internal interface between the context code (xcal_api.cu) and the serving
// loop (xcal_serve.cpp): where a case's device arrays go, and the construction
// of a case as one relocatable device image.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/xcal.h"
#include "xcal_device.cuh"

namespace xcal {

// Destination of a case's device arrays.  An ordinary context allocates and
// uploads each array on its stream; the serving loop lays the arrays out in
// one region of its device arena, with the initialised part staged in pinned
// host memory that the serving kernel copies in itself.
struct Sink {
  virtual ~Sink() {}
  virtual void *put(const void *src, size_t bytes) = 0;   // initialised from host data
  virtual void *zeros(size_t bytes) = 0;                  // initialised to zero
  virtual void *scratch(size_t bytes) = 0;                // contents undefined
  virtual bool ok() const = 0;
  virtual int error() const { return XCAL_ERR_OOM; }
  virtual std::string message() const { return "device allocation failed"; }
  template <class T>
  T *put_v(const std::vector<T> &v) {
    return (T *)put(v.empty() ? nullptr : v.data(), sizeof(T) * v.size());
  }
  template <class T>
  T *zeros_n(size_t n) {
    return (T *)zeros(sizeof(T) * (n ? n : 1));
  }
  template <class T>
  T *scratch_n(size_t n) {
    return (T *)scratch(sizeof(T) * (n ? n : 1));
  }
};

// Layout of a case image: [copy | zero | scratch], each part 256-byte
// aligned.  With measure set, only the sizes are computed (the returned
// pointers are not usable); otherwise pointers are dev_base + offset and the
// copy part is written to host_img.
struct ImageSink : Sink {
  static constexpr size_t ALIGN = 256;
  bool measure = true;
  char *dev_base = nullptr;
  char *host_img = nullptr;
  size_t copy_size = 0, zero_size = 0, scratch_size = 0;   // set by the measure pass
  size_t copy_off = 0, zero_off = 0, scratch_off = 0;
  static size_t up(size_t x) { return (x + ALIGN - 1) / ALIGN * ALIGN; }
  void *put(const void *src, size_t bytes) override {
    const size_t off = copy_off;
    copy_off = up(off + (bytes ? bytes : 1));
    if (!measure && src && bytes) std::memcpy(host_img + off, src, bytes);
    return dev_base + off;
  }
  void *zeros(size_t bytes) override {
    const size_t off = zero_off;
    zero_off = up(off + (bytes ? bytes : 1));
    return dev_base + copy_size + off;
  }
  void *scratch(size_t bytes) override {
    const size_t off = scratch_off;
    scratch_off = up(off + (bytes ? bytes : 1));
    return dev_base + copy_size + zero_size + off;
  }
  bool ok() const override { return true; }
  // after a measure pass: fix the part sizes and restart for the build pass
  void finish_measure() {
    copy_size = up(copy_off);
    zero_size = up(zero_off);
    scratch_size = up(scratch_off);
    copy_off = zero_off = scratch_off = 0;
    measure = false;
  }
  size_t total() const { return copy_size + zero_size + scratch_size; }
};

// A case built for the serving kernel: its parameters (device pointers into
// the image) and what the host needs to read its results back.
struct CaseImage {
  KParams prm;
  int ns = 2;
  int64_t n = 0;              // cells
  int ntiles = 0;
  std::vector<int64_t> perm;  // caller cell -> device cell
  std::vector<double> uz;     // z velocity of a 2D case (unchanged by the run)
};

// Builds `cfg` on the mesh `mesh` (host descriptor) into `sink`, with the
// initial fields U0 (3 x n, caller order) and p0: renumbering, layout, BC
// tables, work arrays, run arrays for `iters` iterations.  Runs twice per
// case: a measure pass, then the build pass into the allocated region.
// gmres_ctas: CTAs the GMRES scratch is sized for.
int build_case_image(const xcal_mesh_desc *mesh, int renumber, const xcal_case *cfg, const double *U0,
                     const double *p0, double tolerance, int iters, int gmres_ctas, Sink &sink, CaseImage &out,
                     std::string &err);

}  // namespace xcal
