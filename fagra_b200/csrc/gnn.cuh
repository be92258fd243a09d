// Learned block preconditioner for the reduced camera system: the interface
// the Schur backend uses. The network and its kernels live in gnn.cu.
#pragma once
#include "schur.cuh"
#include "kernels.cuh"
#include <functional>

namespace fg {

// What the Schur backend exposes at one damping: block factors of
// B + lambda I (cameras) and C + lambda I (points) in the Gram layout, the
// reference-layout cross blocks E_e (element (c,p) at (e*pw+p)*cw+c) and the
// edge/incidence maps. `factors` and `cross` hold the storage type (f64 when
// `f64`, else f32).
struct SchurView {
  Layout L;
  const void* factors;
  const void* cross;
  bool f64;
  const DEdgeMeta* edges;
  int64_t nedges;
  const int64_t *pt_edge_off, *pt_edge, *cam_edge_off, *cam_edge;
  const uint8_t* observed;
  double lambda;
  // point-sorted edge records (28 storage words per edge: E_e column-major
  // cw x pw, then the packed camera / point word) in the order of pt_edge, or
  // null when the backend keeps none; with them the features need no cross array
  const void* rec = nullptr;
  // per edge in camera-major order (cam_edge): x = the edge's point-sorted
  // position, y = its point; null when the backend has not built it
  const int2* cam_meta = nullptr;
};

// y = S x for device vectors of the retained length (f64), S at the view's damping.
using ReducedApply = std::function<fg_status(const double* x, double* y)>;

constexpr int GNN_MAX_CW = 9;
constexpr int GNN_MAX_PW = 4;
constexpr int64_t GNN_MAX_CAMERAS = 16384;

fg_status gnn_check(const fg_gnn* g, size_t cw, size_t pw, size_t cameras, int device);
// Overwrites the explicit preconditioner blocks minv (storage type, cw x cw per
// camera) of observed cameras with L^-T (A A^T + eps I) L^-1 from the network;
// *nonfinite counts cameras whose learned block was not finite (they keep the
// block-Jacobi inverse already in minv).
fg_status gnn_precondition(fg_gnn* g, const SchurView& v, void* minv, cudaStream_t st, unsigned* nonfinite);
// Appends one training system built from the view (features, covisibility,
// whitened probes through `apply`); x_dev/y_dev are retained-length f64
// scratch. kind 0: Gaussian x_hat and `apply` = S; kind 1: Gaussian y_hat and
// `apply` = S^-1 (a converged reduced solve).
fg_status gnn_capture(fg_gnn* g, const SchurView& v, size_t probes, uint64_t seed, int kind,
                      const ReducedApply& apply, double* x_dev, double* y_dev, cudaStream_t st, size_t* index);

}  // namespace fg
