// Schur backend host orchestration: fagra's `Schur` (src/schur.rs) with all
// numerical work on the device. Host code only validates emissions, stages
// them (src/linear_model.rs:180-210 packing) and builds integer index maps.
#include "kernels.cuh"
#include "camside.cuh"
#include "fastpath.cuh"
#include "setup.cuh"
#include "sort.cuh"
#include "gnn.cuh"
#include <algorithm>
#include <cstdlib>
#include <map>
#include <mutex>
#include <numeric>
#include <tuple>

namespace fg {

namespace {

// Widths with compiled specializations; other widths (<= MAXW) use runtime loops.
#define FG_DISPATCH_WIDTHS(cw, pw, BODY)                     \
  do {                                                        \
    if ((cw) == 9 && (pw) == 3) { constexpr int CW_ = 9, PW_ = 3; BODY; }      \
    else if ((cw) == 6 && (pw) == 3) { constexpr int CW_ = 6, PW_ = 3; BODY; } \
    else if ((cw) == 2 && (pw) == 2) { constexpr int CW_ = 2, PW_ = 2; BODY; } \
    else if ((cw) == 1 && (pw) == 1) { constexpr int CW_ = 1, PW_ = 1; BODY; } \
    else { constexpr int CW_ = 0, PW_ = 0; BODY; }                             \
  } while (0)

template <class T>
struct TypeTag {};

// For the learned preconditioner's camera pass: every edge's index in the
// camera-major order (cam_edge), then, point-major, each edge's point-sorted
// position and point index at that index, so the pass reads one coalesced
// int2 per edge instead of gathering the edge's position and metadata.
// The loop condition of the single-launch PCG graph (a WHILE node whose body
// is a fixed number of iterations): continue while the solve runs (mixed
// precision: until done == 1, so a pending FP64 verdict keeps it going) and
// fewer trips than the iteration limit allows have run, the same bound as the
// polling loop's (max_iterations + 8 launched iterations).
__global__ void k_pcg_continue(cudaGraphConditionalHandle h, PcgState* st, int mixed, unsigned iters_per_trip) {
  const bool running = mixed ? st->done != 1 : st->done == 0;
  const unsigned trips = ++st->trips;
  const unsigned long long limit = ((unsigned long long)st->max_iterations + 8 + iters_per_trip - 1) / iters_per_trip;
  cudaGraphSetConditional(h, running && trips < limit ? 1u : 0u);
}

__global__ void k_cam_rank(int64_t nedges, const int64_t* cam_edge, int32_t* rank) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k < nedges) rank[cam_edge[k]] = (int32_t)k;
}
__global__ void k_cam_meta(int64_t nedges, const int64_t* pt_edge, const DEdgeMeta* edges, const int32_t* rank,
                           int2* meta) {
  const int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < nedges) {
    const int64_t e = pt_edge[j];
    meta[rank[e]] = make_int2((int32_t)j, edges[e].pt);
  }
}

}  // namespace

template <class TS>
class SchurImpl final : public Backend {
 public:
  // ---- configuration (src/schur.rs:116-143)
  fg_schur_options opt;
  size_t retained, cw, pw;
  int dev;
  cudaStream_t st = nullptr;
  int nsm = 148;

  // ---- prepared sizes
  size_t dim = 0, nC = 0, nP = 0;
  bool ready = false;

  // ---- statistics / diagnostics
  size_t solves = 0, iterations = 0;
  fg_schur_diagnostics diag{};
  fg_schur_timings tim{};

  // ---- host staging for generic emissions (LinearizedModel layout)
  std::vector<HostBlock> h_blocks;
  std::vector<double> h_values, h_negres;
  std::vector<HostEdge> h_edges;
  size_t h_rows = 0;
  // structure of the last upload (to skip rebuilding identical index maps)
  std::vector<HostBlock> up_blocks;
  std::vector<HostEdge> up_edges;
  size_t up_rows = 0;
  bool structure_valid = false;
  bool pure_pairs = false;     // every emission is exactly one camera-point edge
  // The device BAL layout: emission k is one camera-point edge with rows 2k,
  // 2k+1 and values [24k, 24k+24) (camera 2x9, then point 2x3).
  bool bal_layout() const { return source == DEVICE_BAL && pure_pairs && cw == 9 && pw == 3; }
  DBuf<double> d_raw;  // BAL layout: raw Gram blocks (45 per camera, 6 per point) of the current model
  DBuf<double> d_inv_scales;  // BAL layout: 1 / column scale
  bool cross_current = false;  // d_cross holds this linearization's cross blocks

  // ---- model source
  enum Source { NONE, HOST, DEVICE_BAL, DEVICE_PAIRS } source = NONE;
  // device pair batches (accumulate_pairs): emissions so far, their rows and
  // values, per-emission variables / first row / first value / rows, and the
  // variables and rows of the structure built last (to reuse it)
  size_t dp_em = 0, dp_rows = 0, dp_vals = 0, dp_built = 0;
  DBuf<uint32_t> d_em_cam, d_em_pt, d_em_prev;
  DBuf<int64_t> d_em_row, d_em_val;
  DBuf<int32_t> d_em_rows;
  DBuf<int> d_dp_flags;
  HBuf<int> h_dp_flags;
  bool device_model_current = false;  // device values/negres are current
  bool gradient_current = false;
  uint64_t bal_bound = 0;             // id of the BAL structure currently bound
  size_t bal_obs = 0;

  // ---- device model and index maps
  size_t rows = 0, nblocks = 0, nedges = 0, nvalues = 0, nemissions = 0;
  DBuf<DBlockMeta> d_blocks;
  DBuf<DEdgeMeta> d_edges;
  DBuf<int64_t> d_var_off, d_var_blk, d_pt_edge_off, d_pt_edge, d_cam_edge_off, d_cam_edge, d_emi_off;
  DBuf<uint8_t> d_observed;
  std::vector<uint8_t> h_observed;
  // camera-major (point-sorted position, point) per edge, built on first use
  // after each structure build (ensure_cam_meta)
  DBuf<int2> d_cam_meta;
  DBuf<int32_t> d_cam_rank;
  bool cam_meta_ok = false;
  DBuf<TS> d_values;
  DBuf<double> d_negres;

  // ---- numerics
  DBuf<double> d_g, d_scales, d_work, d_rhs, d_zred, d_step, d_tmpd, d_qd, d_jd, d_camjt;
  DBuf<TS> d_gram, d_factors, d_precond, d_cross, d_minv;
  DBuf<TS> d_x, d_r, d_z, d_pp, d_q, d_t;  // PCG vectors in the storage precision
  DBuf<double> d_partials, d_norm;
  DBuf<unsigned> d_counters;
  DBuf<int> d_flags;
  DBuf<PcgState> d_pcg;
  DBuf<VerifyState> d_ver;
  HBuf<double> h_step, h_scalar;
  HBuf<PcgState> h_pcg;
  HBuf<VerifyState> h_ver;
  HBuf<unsigned> h_count;
  FastPath<TS> fast;  // specialized BAL (9,3) single-pass reduced operator
  // learned preconditioner (FG_PRECOND_LEARNED): the attached network, whether
  // the one-time block-Jacobi comparison has run, and whether it switched the
  // network off for this backend
  fg_gnn* learned = nullptr;
  bool learned_compared = false, learned_off = false;
  DBuf<double> d_keep;  // the learned solution while the comparison solve runs
  // two-level PCG (opt.coarse_correction): the problem's coarse basis
  // (unscaled), W = D * basis in f64 and storage precision, S W, and
  // G = (W^T S W)^-1 for the current damping
  double learned_infer_seconds = 0;  // features + network of the comparison solve
  // the FP32 solve ended on an FP64 replacement residual of the z in d_zred
  // (h_pcg holds it), so verification need not recompute S z - b
  bool final_residual_known = false;
  DBuf<uint32_t> d_bal_stage;  // emission orders by camera and by point, and the sorted keys
  SortScratch sort_scratch;
  int nk = 0;
  bool coarse_on = false, basis_scaled = false;
  DBuf<double> d_basis, d_Wd, d_E, d_G;
  DBuf<int> d_coarse_ok;
  DBuf<TS> d_Wt, d_SWt;
  const void* graph_coarse[3] = {nullptr, nullptr, nullptr};  // W, G, on: what the PCG graphs captured

  Layout layout() const {
    Layout L;
    L.retained = (int64_t)retained;
    L.dim = (int64_t)dim;
    L.cw = (int32_t)cw;
    L.pw = (int32_t)pw;
    L.nC = (int32_t)nC;
    L.nP = (int32_t)nP;
    return L;
  }

  SchurImpl(size_t r, size_t c, size_t p, const fg_schur_options& o) : opt(o), retained(r), cw(c), pw(p), dev(o.device) {}
  ~SchurImpl() override { drop_graphs(); }

  fg_status init() {
    FG_TRY(select_device(dev));
    FG_TRY(device_stream(dev, &st));
    nsm = sm_count(dev);
    // FAGRA_B200_POLLED_GRAPHS set when the backend is created: the polled
    // 8-iteration graphs instead of the single-launch conditional graph (the
    // fallback path, selectable so that it stays tested)
    cond_failed = std::getenv("FAGRA_B200_POLLED_GRAPHS") != nullptr;
    FG_TRY(d_pcg.resize(1));
    FG_TRY(d_ver.resize(1));
    FG_TRY(h_pcg.resize(1));
    FG_TRY(h_ver.resize(1));
    FG_TRY(h_count.resize(4));
    FG_TRY(h_scalar.resize(4));
    FG_TRY(d_counters.resize(8));
    FG_TRY(d_flags.resize(4));
    FG_TRY(d_norm.resize(4));
    FG_CUDA(cudaMemsetAsync(d_pcg.get(), 0, sizeof(PcgState), st));
    FG_CUDA(cudaMemsetAsync(d_ver.get(), 0, sizeof(VerifyState), st));
    FG_CUDA(cudaMemsetAsync(d_counters.get(), 0, 8 * sizeof(unsigned), st));
    FG_TRY(d_partials.resize(8 * 65536));
    return FG_OK;
  }

  // ------------------------------------------------------------------ trait
  int kind() const override { return 0; }
  fg_status set_options(const fg_schur_options& o) override {
    if (o.preconditioner < FG_PRECOND_RETAINED_BLOCKS || o.preconditioner > FG_PRECOND_LEARNED) {
      set_error("unknown preconditioner");
      return FG_INVALID_OPTIONS;
    }
    if (o.operator_variant < 0 || o.operator_variant > NVARIANTS) {
      set_error("operator_variant must be 0 (autotune) or 1..4");
      return FG_INVALID_OPTIONS;
    }
    if (o.learned_policy != 0 && o.learned_policy != 1) {
      set_error("learned_policy must be 0 (compare once) or 1 (always)");
      return FG_INVALID_OPTIONS;
    }
    if (o.preconditioner != opt.preconditioner || o.learned_policy != opt.learned_policy)
      learned_compared = learned_off = false;
    if (!o.coarse_correction) nk = 0;
    if (o.operator_variant != opt.operator_variant) fast.tuned = false;
    int keep = dev;
    opt = o;
    opt.device = keep;
    return FG_OK;
  }

  fg_status prepare(size_t dimension) override {  // src/schur.rs:409-431
    ready = false;
    solves = iterations = 0;
    diag = fg_schur_diagnostics{};
    tim = fg_schur_timings{};
    if (cw == 0 || pw == 0 || retained > dimension || retained % cw || (dimension - retained) % pw ||
        opt.max_iterations == 0 || !(opt.relative_tolerance >= 0 && opt.relative_tolerance < 1)) {
      set_error("Schur prepare: invalid partition or controls");
      return FG_INVALID_OPTIONS;
    }
    FG_TRY(select_device(dev));
    // the PCG graphs stay: launch_graph re-captures them if a buffer moves
    if (dimension != dim) structure_valid = false;
    dim = dimension;
    nC = retained / cw;
    nP = (dim - retained) / pw;
    FG_TRY(d_g.resize(dim));
    FG_TRY(d_scales.resize(dim));
    FG_TRY(d_work.resize(dim));
    FG_TRY(d_step.resize(dim));
    FG_TRY(d_tmpd.resize(std::max(dim, (size_t)1)));
    FG_TRY(d_rhs.resize(retained));
    FG_TRY(d_zred.resize(retained));
    FG_TRY(d_qd.resize(retained));
    FG_TRY(d_camjt.resize(retained));
    FG_TRY(h_step.resize(dim));
    FG_TRY(d_x.resize(retained));
    FG_TRY(d_r.resize(retained));
    FG_TRY(d_z.resize(retained));
    FG_TRY(d_pp.resize(retained));
    FG_TRY(d_q.resize(retained));
    FG_TRY(d_t.resize(nP * pw));
    size_t ng = nC * cw * cw + nP * pw * pw;
    FG_TRY(d_gram.resize(ng));
    FG_TRY(d_factors.resize(ng));
    FG_TRY(d_precond.resize(ng));
    FG_TRY(d_minv.resize(std::max<size_t>(nC * cw * cw, 1)));
    FG_TRY(d_observed.resize(nC + nP));
    return clear();
  }

  fg_status clear() override {  // src/schur.rs:432-437
    ready = false;
    nk = 0;
    basis_scaled = false;
    h_blocks.clear();
    h_values.clear();
    h_negres.clear();
    h_edges.clear();
    h_rows = 0;
    source = HOST;
    dp_em = dp_rows = dp_vals = 0;
    device_model_current = false;
    gradient_current = false;
    return FG_OK;
  }

  // A device batch of bipartite emissions (k_pairs_pack), appended after the
  // batches since the last clear; emission order = batch order, then k.
  fg_status accumulate_pairs(size_t count, size_t prow, const uint32_t* cam, const uint32_t* pt, const double* r,
                             const double* jr, const double* je) override {
    ready = false;
    if (source != DEVICE_PAIRS) {
      FG_TRY(clear());
      source = DEVICE_PAIRS;
    }
    if (count == 0) return FG_OK;
    if (!cam || !pt || !r || !jr || !je) return FG_NULL_ARGUMENT;
    if (prow == 0 || prow > (size_t)MAXW) {
      set_error("device emission batches take 1..16 rows per emission");
      return FG_DIMENSION_MISMATCH;
    }
    if (nC == 0 || nP == 0) {
      set_error("device emission batches need retained and eliminated variables");
      return FG_UNSUPPORTED_STRUCTURE;
    }
    FG_TRY(select_device(dev));
    const size_t em = dp_em + count, nr = dp_rows + count * prow, nv = dp_vals + count * prow * (cw + pw);
    FG_TRY(d_em_cam.grow_keep(em, dp_em, st));
    FG_TRY(d_em_pt.grow_keep(em, dp_em, st));
    FG_TRY(d_em_row.grow_keep(em, dp_em, st));
    FG_TRY(d_em_val.grow_keep(em, dp_em, st));
    FG_TRY(d_em_rows.grow_keep(em, dp_em, st));
    FG_TRY(d_negres.grow_keep(nr, dp_rows, st));
    FG_TRY(d_values.grow_keep(nv, dp_vals, st));
    FG_TRY(d_dp_flags.resize(2));
    FG_TRY(h_dp_flags.resize(2));
    FG_CUDA(cudaMemsetAsync(d_dp_flags.get(), 0, 2 * sizeof(int), st));
    FG_LAUNCH(k_pairs_pack<TS>, grid_for(count, 128), 128, 0, st, (int64_t)count, (int)prow, (int)cw, (int)pw,
              (int64_t)nC, (int64_t)nP, cam, pt, r, jr, je, (int64_t)dp_em, (int64_t)dp_rows, (int64_t)dp_vals,
              d_em_cam.get(), d_em_pt.get(), d_em_row.get(), d_em_val.get(), d_em_rows.get(), d_negres.get(),
              d_values.get(), d_dp_flags.get());
    FG_CUDA(cudaMemcpyAsync(h_dp_flags.get(), d_dp_flags.get(), 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    if (h_dp_flags.get()[0]) {  // src/optimization.rs:575-584: a variable outside the layout
      set_error("device emission batch: a variable index outside the layout");
      return FG_INVALID_EMISSION;
    }
    if (h_dp_flags.get()[1]) {  // src/optimization.rs:556-558, 596-598
      set_error("device emission batch: nonfinite residual or Jacobian");
      return FG_INVALID_EVALUATION;
    }
    dp_em = em;
    dp_rows = nr;
    dp_vals = nv;
    device_model_current = false;
    gradient_current = false;
    return FG_OK;
  }

  // The maps build_structure derives, for the device pair emissions: as
  // build_structure_bal with the emissions' own rows, widths and starts.
  fg_status build_structure_pairs() {
    const size_t obs = dp_em;
    rows = dp_rows;
    nblocks = 2 * obs;
    nedges = obs;
    const size_t nvar = nC + nP;
    if (nC >= ((size_t)1 << 31) || nP >= ((size_t)1 << 31)) return FG_UNSUPPORTED_STRUCTURE;
    FG_TRY(d_bal_stage.resize(std::max<size_t>(4 * obs, 1)));  // cam_order | pt_order | sorted cams | sorted points
    uint32_t* stage = d_bal_stage.get();
    FG_TRY(d_cam_edge_off.resize(nC + 1));
    FG_TRY(d_pt_edge_off.resize(nP + 1));
    FG_TRY(d_var_off.resize(nvar + 1));
    FG_TRY(d_observed.resize(std::max<size_t>(nvar, 1)));
    FG_TRY(stable_order(d_em_cam.get(), obs, (uint32_t)nC, stage, stage + 2 * obs, sort_scratch, st));
    FG_TRY(key_offsets(stage + 2 * obs, obs, (uint32_t)nC, d_cam_edge_off.get(), st));
    FG_TRY(stable_order(d_em_pt.get(), obs, (uint32_t)nP, stage + obs, stage + 3 * obs, sort_scratch, st));
    FG_TRY(key_offsets(stage + 3 * obs, obs, (uint32_t)nP, d_pt_edge_off.get(), st));
    FG_TRY(d_blocks.resize(std::max<size_t>(nblocks, 1)));
    FG_TRY(d_edges.resize(std::max<size_t>(nedges, 1)));
    FG_TRY(d_var_blk.resize(std::max<size_t>(nblocks, 1)));
    FG_TRY(d_cam_edge.resize(std::max<size_t>(nedges, 1)));
    FG_TRY(d_pt_edge.resize(std::max<size_t>(nedges, 1)));
    FG_TRY(d_emi_off.resize(obs + 1));
    FG_LAUNCH(k_pairs_structure, grid_for(obs + 1, 256), 256, 0, st, (int64_t)obs, (int64_t)retained, (int)cw,
              (int)pw, d_em_cam.get(), d_em_pt.get(), d_em_row.get(), d_em_val.get(), d_em_rows.get(), stage,
              stage + obs, d_blocks.get(), d_edges.get(), d_var_blk.get(), d_cam_edge.get(), d_pt_edge.get(),
              d_emi_off.get());
    FG_LAUNCH(k_bal_var_offsets, grid_for(nvar + 1, 256), 256, 0, st, (int64_t)nC, (int64_t)nP, (int64_t)obs,
              d_cam_edge_off.get(), d_pt_edge_off.get(), d_var_off.get(), d_observed.get());
    h_observed.resize(nvar);
    if (nvar) FG_CUDA(cudaMemcpyAsync(h_observed.data(), d_observed.get(), nvar, cudaMemcpyDeviceToHost, st));
    nemissions = obs;
    pure_pairs = obs > 0;
    FG_TRY(d_cross.resize(std::max<size_t>(nedges * cw * pw, 1)));
    FG_TRY(d_jd.resize(std::max<size_t>(rows, 1)));
    // remember what this structure was built from (cameras | points | rows)
    FG_TRY(d_em_prev.resize(std::max<size_t>(3 * obs, 1)));
    if (obs) {
      FG_CUDA(cudaMemcpyAsync(d_em_prev.get(), d_em_cam.get(), obs * sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
      FG_CUDA(cudaMemcpyAsync(d_em_prev.get() + obs, d_em_pt.get(), obs * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                              st));
      FG_CUDA(cudaMemcpyAsync(d_em_prev.get() + 2 * obs, d_em_rows.get(), obs * sizeof(uint32_t),
                              cudaMemcpyDeviceToDevice, st));
    }
    dp_built = obs;
    FG_CUDA(cudaStreamSynchronize(st));
    structure_valid = true;
    fast.invalidate();
    cam_meta_ok = false;
    drop_graphs();
    return FG_OK;
  }

  // Whether the pair emissions are the ones the current structure was built
  // from (same variables and rows in the same order).
  fg_status same_pairs(bool* same) {
    *same = false;
    if (!structure_valid || bal_bound || !up_blocks.empty() || dp_built != dp_em || dp_em == 0) return FG_OK;
    FG_TRY(d_dp_flags.resize(2));
    FG_TRY(h_dp_flags.resize(2));
    FG_CUDA(cudaMemsetAsync(d_dp_flags.get(), 0, sizeof(int), st));
    FG_LAUNCH(k_pairs_differ, grid_for(dp_em, 256), 256, 0, st, (int64_t)dp_em, d_em_cam.get(), d_em_pt.get(),
              (const uint32_t*)d_em_rows.get(), d_em_prev.get(), d_dp_flags.get());
    FG_CUDA(cudaMemcpyAsync(h_dp_flags.get(), d_dp_flags.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    *same = h_dp_flags.get()[0] == 0;
    return FG_OK;
  }

  fg_status accumulate(size_t nrows, const double* r, size_t nb, const size_t* bcols, const size_t* widths,
                       const double* const* jac, const ptrdiff_t* rs, const ptrdiff_t* cs) override {
    // src/schur.rs:438-482 structure validation, then LinearizedModel packing.
    ready = false;
    if (source != HOST) clear();
    if (nrows && !r) return FG_NULL_ARGUMENT;
    if (nb && (!bcols || !widths || !jac || !rs || !cs)) return FG_NULL_ARGUMENT;
    bool has_l = false, has_r = false;
    size_t lcol = 0, lidx = 0, rcol = 0, ridx = 0;
    size_t start = h_blocks.size();
    for (size_t i = 0; i < nb; ++i) {
      size_t col = bcols[i], end = col + widths[i];
      if (end < col || end > dim) return FG_DIMENSION_MISMATCH;
      if (col < retained) {
        if (col % cw || widths[i] != cw || end > retained || has_l) return FG_UNSUPPORTED_STRUCTURE;
        has_l = true; lcol = col; lidx = start + i;
      } else {
        if ((col - retained) % pw || widths[i] != pw || has_r) return FG_UNSUPPORTED_STRUCTURE;
        has_r = true; rcol = col - retained; ridx = start + i;
      }
      if (widths[i] && nrows && !jac[i]) return FG_NULL_ARGUMENT;
    }
    size_t row = h_rows;
    h_rows += nrows;
    for (size_t i = 0; i < nrows; ++i) h_negres.push_back(-r[i]);
    for (size_t b = 0; b < nb; ++b) {
      h_blocks.push_back({row, bcols[b], nrows, widths[b], h_values.size()});
      for (size_t j = 0; j < widths[b]; ++j)
        for (size_t i = 0; i < nrows; ++i) h_values.push_back(jac[b][(ptrdiff_t)i * rs[b] + (ptrdiff_t)j * cs[b]]);
    }
    if (has_l && has_r) h_edges.push_back({lcol, rcol, lidx, ridx});
    device_model_current = false;
    gradient_current = false;
    return FG_OK;
  }

  // Build and upload index maps for a structure (host integer bookkeeping).
  fg_status build_structure(const std::vector<HostBlock>& blocks, const std::vector<HostEdge>& edges, size_t nrows) {
    dp_built = 0;
    rows = nrows;
    nblocks = blocks.size();
    nedges = edges.size();
    size_t nvar = nC + nP;
    std::vector<DBlockMeta> mb(nblocks);
    std::vector<int64_t> var_of(nblocks), var_off(nvar + 1, 0), var_blk(nblocks);
    for (size_t i = 0; i < nblocks; ++i) {
      const HostBlock& b = blocks[i];
      mb[i] = {(int64_t)b.row, (int64_t)b.start, (int64_t)b.col, (int32_t)b.rows, (int32_t)b.cols};
      int64_t v = b.col < retained ? (int64_t)(b.col / cw) : (int64_t)(nC + (b.col - retained) / pw);
      var_of[i] = b.cols ? v : -1;
      if (b.cols) var_off[v + 1]++;
    }
    for (size_t v = 0; v < nvar; ++v) var_off[v + 1] += var_off[v];
    {
      std::vector<int64_t> fill(var_off.begin(), var_off.end() - 1);
      for (size_t i = 0; i < nblocks; ++i)
        if (var_of[i] >= 0) var_blk[fill[var_of[i]]++] = (int64_t)i;
    }
    h_observed.assign(nvar, 0);
    for (size_t v = 0; v < nvar; ++v) h_observed[v] = var_off[v + 1] > var_off[v];
    std::vector<DEdgeMeta> me(nedges);
    std::vector<int64_t> pt_off(nP + 1, 0), cam_off(nC + 1, 0), pt_e(nedges), cam_e(nedges);
    for (size_t e = 0; e < nedges; ++e) {
      me[e] = {(int32_t)(edges[e].retained / cw), (int32_t)(edges[e].eliminated / pw), (int64_t)edges[e].lblk,
               (int64_t)edges[e].rblk};
      pt_off[me[e].pt + 1]++;
      cam_off[me[e].cam + 1]++;
    }
    for (size_t p = 0; p < nP; ++p) pt_off[p + 1] += pt_off[p];
    for (size_t c = 0; c < nC; ++c) cam_off[c + 1] += cam_off[c];
    {
      std::vector<int64_t> fp(pt_off.begin(), pt_off.end() - 1), fc(cam_off.begin(), cam_off.end() - 1);
      for (size_t e = 0; e < nedges; ++e) {
        pt_e[fp[me[e].pt]++] = (int64_t)e;
        cam_e[fc[me[e].cam]++] = (int64_t)e;
      }
    }
    // emissions: consecutive blocks sharing a row start
    std::vector<int64_t> emi;
    for (size_t i = 0; i < nblocks; ++i)
      if (i == 0 || blocks[i].row != blocks[i - 1].row || blocks[i].rows == 0) emi.push_back((int64_t)i);
    emi.push_back((int64_t)nblocks);
    nemissions = emi.size() - 1;
    pure_pairs = nedges > 0 && nblocks == 2 * nedges && nemissions == nedges;
    FG_TRY(upload(d_blocks, mb.data(), mb.size(), st));
    FG_TRY(upload(d_edges, me.data(), me.size(), st));
    FG_TRY(upload(d_var_off, var_off.data(), var_off.size(), st));
    FG_TRY(upload(d_var_blk, var_blk.data(), var_blk.size(), st));
    FG_TRY(upload(d_pt_edge_off, pt_off.data(), pt_off.size(), st));
    FG_TRY(upload(d_pt_edge, pt_e.data(), pt_e.size(), st));
    FG_TRY(upload(d_cam_edge_off, cam_off.data(), cam_off.size(), st));
    FG_TRY(upload(d_cam_edge, cam_e.data(), cam_e.size(), st));
    FG_TRY(upload(d_emi_off, emi.data(), emi.size(), st));
    FG_TRY(upload(d_observed, h_observed.data(), h_observed.size(), st));
    FG_TRY(d_cross.resize(std::max<size_t>(nedges * cw * pw, 1)));
    FG_TRY(d_jd.resize(std::max<size_t>(rows, 1)));
    // synchronize so host vectors may be released safely
    FG_CUDA(cudaStreamSynchronize(st));
    structure_valid = true;
    fast.invalidate();
    cam_meta_ok = false;
    drop_graphs();
    return FG_OK;
  }

  // The maps build_structure derives, for the BAL emission layout, built on
  // the device: stable orders of the emissions by camera and by point (radix
  // sorts), their offsets, then every map in one pass over the emissions.
  fg_status build_structure_bal(size_t cams, size_t pts, size_t obs, const uint32_t* ocam, const uint32_t* opt) {
    dp_built = 0;
    rows = 2 * obs;
    nblocks = 2 * obs;
    nedges = obs;
    const size_t nvar = nC + nP;
    if (cams >= ((size_t)1 << 32) || pts >= ((size_t)1 << 32)) return FG_UNSUPPORTED_STRUCTURE;
    FG_TRY(d_bal_stage.resize(std::max<size_t>(4 * obs, 1)));  // cam_order | pt_order | sorted cams | sorted points
    uint32_t* stage = d_bal_stage.get();
    FG_TRY(d_cam_edge_off.resize(nC + 1));
    FG_TRY(d_pt_edge_off.resize(nP + 1));
    FG_TRY(d_var_off.resize(nvar + 1));
    FG_TRY(d_observed.resize(std::max<size_t>(nvar, 1)));
    FG_TRY(stable_order(ocam, obs, (uint32_t)cams, stage, stage + 2 * obs, sort_scratch, st));
    FG_TRY(key_offsets(stage + 2 * obs, obs, (uint32_t)cams, d_cam_edge_off.get(), st));
    FG_TRY(stable_order(opt, obs, (uint32_t)pts, stage + obs, stage + 3 * obs, sort_scratch, st));
    FG_TRY(key_offsets(stage + 3 * obs, obs, (uint32_t)pts, d_pt_edge_off.get(), st));
    FG_TRY(d_blocks.resize(std::max<size_t>(nblocks, 1)));
    FG_TRY(d_edges.resize(std::max<size_t>(nedges, 1)));
    FG_TRY(d_var_blk.resize(std::max<size_t>(nblocks, 1)));
    FG_TRY(d_cam_edge.resize(std::max<size_t>(nedges, 1)));
    FG_TRY(d_pt_edge.resize(std::max<size_t>(nedges, 1)));
    FG_TRY(d_emi_off.resize(obs + 1));
    FG_LAUNCH(k_bal_structure, grid_for(obs + 1, 256), 256, 0, st, (int64_t)obs, (int64_t)cams, ocam, opt, stage,
              stage + obs, d_blocks.get(), d_edges.get(), d_var_blk.get(), d_cam_edge.get(), d_pt_edge.get(),
              d_emi_off.get());
    FG_LAUNCH(k_bal_var_offsets, grid_for(nvar + 1, 256), 256, 0, st, (int64_t)nC, (int64_t)nP, (int64_t)obs,
              d_cam_edge_off.get(), d_pt_edge_off.get(), d_var_off.get(), d_observed.get());
    h_observed.resize(nvar);
    if (nvar)
      FG_CUDA(cudaMemcpyAsync(h_observed.data(), d_observed.get(), nvar, cudaMemcpyDeviceToHost, st));
    nemissions = obs;
    pure_pairs = obs > 0;
    FG_TRY(d_cross.resize(std::max<size_t>(nedges * cw * pw, 1)));
    FG_TRY(d_jd.resize(std::max<size_t>(rows, 1)));
    FG_CUDA(cudaStreamSynchronize(st));
    structure_valid = true;
    fast.invalidate();
    cam_meta_ok = false;
    drop_graphs();
    return FG_OK;
  }

  static bool same_blocks(const std::vector<HostBlock>& a, const std::vector<HostBlock>& b) {
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); ++i)
      if (a[i].row != b[i].row || a[i].col != b[i].col || a[i].rows != b[i].rows || a[i].cols != b[i].cols ||
          a[i].start != b[i].start)
        return false;
    return true;
  }
  static bool same_edges(const std::vector<HostEdge>& a, const std::vector<HostEdge>& b) {
    if (a.size() != b.size()) return false;
    for (size_t i = 0; i < a.size(); ++i)
      if (a[i].retained != b[i].retained || a[i].eliminated != b[i].eliminated || a[i].lblk != b[i].lblk ||
          a[i].rblk != b[i].rblk)
        return false;
    return true;
  }

  // Upload host emissions and compute the gradient on the device.
  fg_status sync_model() {
    if (source == HOST && !device_model_current) {
      if (!structure_valid || bal_bound || up_rows != h_rows || !same_blocks(up_blocks, h_blocks) ||
          !same_edges(up_edges, h_edges)) {
        bal_bound = 0;
        FG_TRY(build_structure(h_blocks, h_edges, h_rows));
        up_blocks = h_blocks;
        up_edges = h_edges;
        up_rows = h_rows;
      }
      nvalues = h_values.size();
      FG_TRY(d_values.resize(std::max<size_t>(nvalues, 1)));
      if (nvalues) {
        if (std::is_same<TS, double>::value) {
          FG_CUDA(cudaMemcpyAsync(d_values.get(), h_values.data(), nvalues * sizeof(double), cudaMemcpyHostToDevice, st));
        } else {
          std::vector<TS> conv(h_values.begin(), h_values.end());
          FG_CUDA(cudaMemcpyAsync(d_values.get(), conv.data(), nvalues * sizeof(TS), cudaMemcpyHostToDevice, st));
          FG_CUDA(cudaStreamSynchronize(st));
        }
      }
      FG_TRY(upload(d_negres, h_negres.data(), h_negres.size(), st));
      if (d_negres.cap == 0) FG_TRY(d_negres.resize(1));
      FG_CUDA(cudaStreamSynchronize(st));
      device_model_current = true;
      gradient_current = false;
    }
    if (source == DEVICE_PAIRS && !device_model_current) {
      bool same = false;
      FG_TRY(same_pairs(&same));
      if (!same) {
        bal_bound = 0;
        up_blocks.clear();
        up_edges.clear();
        FG_TRY(build_structure_pairs());
      }
      nvalues = dp_vals;
      rows = dp_rows;
      device_model_current = true;
      gradient_current = false;
    }
    if (source == NONE) return FG_INVALID_OPTIONS;
    if (!gradient_current && bal_layout()) {
      // the gradient and the raw Gram blocks (for the column scales) in one pass
      FG_TRY(d_raw.resize(45 * nC + 6 * nP + 1));
      if (nC)
        FG_LAUNCH((k_bal_cam_pass<TS, BAL_MOMENTS>), (unsigned)nC, BAL_CAM_THREADS, 0, st, (int64_t)nC, d_cam_edge_off.get(),
                  d_values.get(), d_negres.get(), (const double*)nullptr, d_g.get(), d_raw.get());
      if (nP)
        FG_LAUNCH(k_bal_point_moments<TS>, grid_for(nP, 128), 128, 0, st, (int64_t)nP, (int64_t)retained,
                  d_pt_edge_off.get(), d_pt_edge.get(), d_values.get(), d_negres.get(), d_g.get(),
                  d_raw.get() + 45 * nC);
      gradient_current = true;
    }
    if (!gradient_current) {
      Layout L = layout();
      if (nC) {
        FG_DISPATCH_WIDTHS(cw, pw, {
          FG_LAUNCH((k_cam_jt_block<CW_, TS, CAM_GRADIENT>), (unsigned)nC, 128, 0, st, L, d_var_off.get(),
                    d_var_blk.get(), d_blocks.get(), d_values.get(), d_negres.get(), (const double*)nullptr, d_g.get());
        });
      }
      if (dim > retained)
        FG_LAUNCH(k_gradient<TS>, grid_for(dim - retained, NT), NT, 0, st, L, (int64_t)retained, d_var_off.get(),
                  d_var_blk.get(), d_blocks.get(), d_values.get(), d_negres.get(), d_g.get());
      gradient_current = true;
    }
    return FG_OK;
  }

  // max |x| over a device array; returns INVALID_EVALUATION on nonfinite.
  template <class T>
  fg_status device_norm_inf(const T* x, size_t n, double* out) {
    if (n == 0) { *out = 0; return FG_OK; }
    unsigned g = std::min<unsigned>(grid_for(n, NT), 4 * nsm);
    FG_LAUNCH(k_norm_inf<T>, g, NT, 0, st, (int64_t)n, x, d_partials.get(), d_counters.get() + 3, d_norm.get());
    FG_CUDA(cudaMemcpyAsync(h_scalar.get(), d_norm.get(), 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    if (h_scalar.get()[1] != 0) {
      set_error("nonfinite value");
      return FG_INVALID_EVALUATION;
    }
    *out = h_scalar.get()[0];
    return FG_OK;
  }

  fg_status gradient_norm(double* out) override {  // src/schur.rs:483-485
    FG_TRY(sync_model());
    return device_norm_inf(d_g.get(), dim, out);
  }

  fg_status prepare_damping(double floor) override {  // src/schur.rs:490-526
    basis_scaled = false;  // new column scales
    ready = false;
    EventTimer tm;
    if (opt.collect_timings) tm.start(st);
    if (!std::isfinite(floor) || floor <= 0) {
      set_error("min_column_norm must be finite and positive");
      return FG_INVALID_OPTIONS;
    }
    FG_TRY(sync_model());
    Layout L = layout();
    int* bad = d_flags.get();
    FG_CUDA(cudaMemsetAsync(bad, 0, 2 * sizeof(int), st));
    if (bal_layout()) {  // from the raw moments sync_model computed with the gradient
      FG_TRY(d_inv_scales.resize(std::max<size_t>(dim, 1)));
      if (nC + nP)
        FG_LAUNCH(k_bal_scales_gram<TS>, grid_for(nC + nP, 128), 128, 0, st, (int64_t)nC, (int64_t)nP, d_raw.get(),
                  d_raw.get() + 45 * nC, floor, d_scales.get(), d_inv_scales.get(), d_gram.get(), bad);
    } else if (nC) {
      FG_CUDA(cudaMemsetAsync(d_gram.get(), 0, nC * cw * cw * sizeof(TS), st));
      FG_DISPATCH_WIDTHS(cw, pw, {
        FG_LAUNCH((k_cam_scales_gram<CW_, TS>), (unsigned)nC, 128, 0, st, L, d_var_off.get(), d_var_blk.get(),
                  d_blocks.get(), d_values.get(), floor, d_scales.get(), d_gram.get(), bad);
      });
    }
    if (nP && !bal_layout()) {
      FG_DISPATCH_WIDTHS(cw, pw, {
        FG_LAUNCH((k_point_scales_gram<PW_, TS>), grid_for(nP, 128), 128, 0, st, L, d_var_off.get(),
                  d_var_blk.get(), d_blocks.get(), d_values.get(), floor, d_scales.get(), d_gram.get(), bad);
      });
    }
    if (nedges) {
      if (fast.ready_for(*this)) {
        // the reference-layout cross array is only needed by the generic
        // right-hand side / back-substitution and the Schur-diagonal factor
        cross_current = !pure_pairs || opt.preconditioner == FG_PRECOND_SCHUR_DIAGONAL ||
                        (learned_active() && !(cw == 9 && pw == 3));  // the 9/3 features read the records
        if (bal_layout())
          FG_LAUNCH(k_edge_records_bal<TS>, grid_for(nedges, REC_T), REC_T, 0, st, (int64_t)nedges,
                    (int64_t)retained, d_pt_edge.get(), d_edges.get(), d_values.get(), d_inv_scales.get(),
                    fast.d_lp.get(), fast.d_erec.get(), cross_current ? d_cross.get() : (TS*)nullptr, bad + 1);
        else
          FG_LAUNCH(k_edge_records2<TS>, grid_for(nedges, REC_T), REC_T, 0, st, (int64_t)nedges, d_pt_edge.get(),
                    d_edges.get(), d_blocks.get(), d_values.get(), d_scales.get(), fast.d_lp.get(), fast.d_erec.get(),
                    cross_current ? d_cross.get() : (TS*)nullptr, bad + 1);
        fast.on = true;
      } else {
        fast.on = false;
        cross_current = true;
        FG_LAUNCH(k_cross<TS>, grid_for(nedges * cw * pw, NT), NT, 0, st, (int64_t)nedges, (int)cw, (int)pw,
                  d_edges.get(), d_blocks.get(), d_values.get(), d_scales.get(), d_cross.get(), bad + 1);
      }
    } else {
      fast.on = false;
    }
    FG_CUDA(cudaMemcpyAsync(h_count.get(), bad, 2 * sizeof(int), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    if (h_count.get()[0] || h_count.get()[1]) {
      fast.on = false;
      set_error("nonfinite column norm or cross block");
      return FG_INVALID_EVALUATION;
    }
    ready = true;
    FG_TRY(autotune_operator());
    if (opt.collect_timings) tim.preparation += tm.stop(st);
    return FG_OK;
  }

  fg_status set_coarse_basis(const double* basis, int k) override {
    if (!opt.coarse_correction || k <= 0) return FG_OK;
    if (k > MAXK) {
      set_error("a coarse basis holds at most 8 vectors");
      return FG_INVALID_OPTIONS;
    }
    FG_TRY(d_basis.resize((size_t)k * std::max<size_t>(retained, 1)));
    if (retained)
      FG_CUDA(cudaMemcpyAsync(d_basis.get(), basis, (size_t)k * retained * sizeof(double), cudaMemcpyDeviceToDevice,
                              st));
    nk = k;
    basis_scaled = false;
    return FG_OK;
  }

  // W = D * basis once the column scales of this linearization exist.
  fg_status scale_basis() {
    if (!nk || basis_scaled || !retained) return FG_OK;
    const size_t n = (size_t)nk * retained;
    FG_TRY(d_Wd.resize(n));
    FG_TRY(d_Wt.resize(n));
    FG_TRY(d_SWt.resize(n));
    FG_TRY(d_E.resize(MAXK * MAXK));
    FG_TRY(d_G.resize(MAXK * MAXK));
    FG_TRY(d_coarse_ok.resize(1));
    FG_LAUNCH(k_coarse_scale<TS>, grid_for(n, 256), 256, 0, st, (int64_t)retained, nk, d_basis.get(), d_scales.get(),
              d_Wd.get(), d_Wt.get());
    basis_scaled = true;
    return FG_OK;
  }

  // G = (W^T S W)^-1 at lambda (nk reduced-operator applications); the
  // two-level preconditioner stays off for this solve if W^T S W is not SPD,
  // and above COARSE_MAX_DAMPING, where damping has already lifted the coarse
  // modes into the block-Jacobi bulk (measured on BAL: 10 -> 13 iterations at
  // lambda = 1, 50 -> 22 at 1e-4).
  static constexpr double COARSE_MAX_DAMPING = 0.1;
  fg_status prepare_coarse(double lambda) {
    coarse_on = false;
    if (!opt.coarse_correction || !nk || !retained || lambda > COARSE_MAX_DAMPING) return sync_graph_coarse();
    FG_TRY(scale_basis());
    if (fast.enabled() && nk == 7) {
      // one pass over the edge records (BAL shape, the 7 gauge vectors)
      FG_TRY(fast.coarse_gram(*this, lambda, d_Wd.get(), nk, d_E.get()));
    } else {
      // S W in the storage precision (the operator the PCG itself applies);
      // the Gram W^T (S W) accumulates in f64
      for (int j = 0; j < nk; ++j) {
        PView<TS> pv{d_Wt.get() + (size_t)j * retained, nullptr, nullptr};
        FG_TRY(apply_reduced<TS>(pv, lambda, lambda, true, d_t.get(), d_SWt.get() + (size_t)j * retained, nullptr,
                                 nullptr));
      }
      FG_LAUNCH(k_coarse_gram<TS>, (unsigned)(nk * nk), 256, 0, st, (int64_t)retained, nk, d_Wd.get(),
                (const TS*)d_SWt.get(), d_E.get());
    }
    // G on the device (no host round trip); a non-SPD E gives G = 0, i.e.
    // one-level PCG, and the verification readback reports it
    FG_LAUNCH(k_coarse_factor, 1, 32, 0, st, nk, (const double*)d_E.get(), d_G.get(), d_coarse_ok.get());
    coarse_on = true;
    return sync_graph_coarse();
  }
  // The PCG graphs bake in the kernel variants and the W / G pointers.
  fg_status sync_graph_coarse() {
    const void* now[3] = {coarse_on ? (const void*)d_Wt.get() : nullptr, coarse_on ? (const void*)d_G.get() : nullptr,
                          coarse_on ? (const void*)this : nullptr};
    if (now[0] != graph_coarse[0] || now[1] != graph_coarse[1] || now[2] != graph_coarse[2]) {
      drop_graphs();
      for (int k = 0; k < 3; ++k) graph_coarse[k] = now[k];
    }
    return FG_OK;
  }

  template <class TX>
  fg_status launch_start(const double* b, TX* x, double rel_tol) {
    Layout L = layout();
    const unsigned bw = wide_block(), gw = wide_grid();
    const size_t shm = bw * sizeof(TS);
    PcgState* ps = d_pcg.get();
    FG_DISPATCH_WIDTHS(cw, pw, {
      if (coarse_on)
        FG_LAUNCH((k_pcg_start<CW_, TS, TX, true>), gw, bw, shm, st, L, b, x, d_r.get(), d_z.get(), d_pp.get(),
                  d_minv.get(), d_partials.get(), ps, rel_tol, (const TS*)d_Wt.get(), (const double*)d_G.get(), nk);
      else
        FG_LAUNCH((k_pcg_start<CW_, TS, TX, false>), gw, bw, shm, st, L, b, x, d_r.get(), d_z.get(), d_pp.get(),
                  d_minv.get(), d_partials.get(), ps, rel_tol, (const TS*)nullptr, (const double*)nullptr, 0);
    });
    return launch_coarse_add();
  }
  template <class TX, bool MIXED>
  fg_status launch_update(TX* x) {
    Layout L = layout();
    const unsigned bw = wide_block(), gw = wide_grid();
    const size_t shm = bw * sizeof(TS);
    PcgState* ps = d_pcg.get();
    FG_DISPATCH_WIDTHS(cw, pw, {
      if (coarse_on)
        FG_LAUNCH_PDL((k_update_wide<CW_, TS, TX, MIXED, true>), gw, bw, shm, st, L, x, d_r.get(), d_z.get(),
                      d_pp.get(), d_q.get(), d_minv.get(), d_partials.get(), ps, (const TS*)d_Wt.get(),
                      (const double*)d_G.get(), nk);
      else
        FG_LAUNCH_PDL((k_update_wide<CW_, TS, TX, MIXED, false>), gw, bw, shm, st, L, x, d_r.get(), d_z.get(),
                      d_pp.get(), d_q.get(), d_minv.get(), d_partials.get(), ps, (const TS*)nullptr,
                      (const double*)nullptr, 0);
    });
    return launch_coarse_add();
  }
  fg_status launch_replace() {
    Layout L = layout();
    const unsigned bw = wide_block(), gw = wide_grid();
    const size_t shm = bw * sizeof(TS);
    PcgState* ps = d_pcg.get();
    FG_DISPATCH_WIDTHS(cw, pw, {
      if (coarse_on)
        FG_LAUNCH((k_replace_wide<CW_, TS, true>), gw, bw, shm, st, L, d_rhs.get(), d_qd.get(), d_r.get(), d_z.get(),
                  d_minv.get(), d_partials.get(), ps, (const TS*)d_Wt.get(), (const double*)d_G.get(), nk);
      else
        FG_LAUNCH((k_replace_wide<CW_, TS, false>), gw, bw, shm, st, L, d_rhs.get(), d_qd.get(), d_r.get(),
                  d_z.get(), d_minv.get(), d_partials.get(), ps, (const TS*)nullptr, (const double*)nullptr, 0);
    });
    return launch_coarse_add();
  }
  fg_status launch_coarse_add() {
    if (coarse_on)
      FG_LAUNCH_PDL(k_coarse_add<TS>, grid_for(retained, 256), 256, 0, st, (int64_t)retained, nk,
                    (const TS*)d_Wt.get(), d_pcg.get(), d_z.get());
    return FG_OK;
  }

  bool learned_active() const {
    return opt.preconditioner == FG_PRECOND_LEARNED && learned != nullptr && !learned_off;
  }
  SchurView view_at(double lambda) const {
    SchurView v;
    v.L = layout();
    v.factors = d_factors.get();
    v.cross = d_cross.get();
    v.f64 = std::is_same<TS, double>::value;
    v.edges = d_edges.get();
    v.nedges = (int64_t)nedges;
    v.pt_edge_off = d_pt_edge_off.get();
    v.pt_edge = d_pt_edge.get();
    v.cam_edge_off = d_cam_edge_off.get();
    v.cam_edge = d_cam_edge.get();
    v.observed = d_observed.get();
    v.lambda = lambda;
    v.rec = fast.on && cw == 9 && pw == 3 ? (const void*)fast.d_erec.get() : nullptr;
    v.cam_meta = cam_meta_ok ? d_cam_meta.get() : nullptr;
    return v;
  }
  // The camera-major (position, point) array of the learned preconditioner's
  // BAL-width camera pass: two passes over the edges, once per structure
  // (positions are 32-bit, so larger structures go without it).
  fg_status ensure_cam_meta() {
    if (cam_meta_ok || cw != 9 || pw != 3 || !nedges || nedges > (size_t)INT32_MAX) return FG_OK;
    FG_TRY(d_cam_rank.resize(nedges));
    FG_TRY(d_cam_meta.resize(nedges));
    FG_LAUNCH(k_cam_rank, grid_for(nedges, 256), 256, 0, st, (int64_t)nedges, d_cam_edge.get(), d_cam_rank.get());
    FG_LAUNCH(k_cam_meta, grid_for(nedges, 256), 256, 0, st, (int64_t)nedges, d_pt_edge.get(), d_edges.get(),
              (const int32_t*)d_cam_rank.get(), d_cam_meta.get());
    cam_meta_ok = true;
    return FG_OK;
  }
  // Explicit block-Jacobi (or Schur-diagonal) inverses into d_minv.
  fg_status write_block_inverses(double lambda) {
    Layout L = layout();
    FG_DISPATCH_WIDTHS(cw, pw, {
      FG_LAUNCH((k_precond_inverse<CW_, TS>), grid_for(nC, 64), 64, 0, st, L, d_observed.get(), precond_factors(),
                lambda, d_minv.get());
    });
    return FG_OK;
  }

  // Factor B and C blocks (+ the optional S_cc preconditioner) for lambda;
  // with `learned_blocks` the attached network then reshapes the inverses.
  fg_status factor(double lambda, unsigned* fallbacks, bool learned_blocks = false) {
    Layout L = layout();
    FG_CUDA(cudaMemsetAsync(d_counters.get() + 4, 0, sizeof(unsigned), st));
    FG_DISPATCH_WIDTHS(cw, pw, {
      if (nC) FG_LAUNCH((k_factor<CW_, TS>), grid_for(nC, 128), 128, 0, st, L, (int64_t)0, (int64_t)nC, (int)cw,
                        d_observed.get(), d_gram.get(), d_factors.get(), lambda, d_counters.get() + 4);
      if (nP) FG_LAUNCH((k_factor<PW_, TS>), grid_for(nP, 128), 128, 0, st, L, (int64_t)nC, (int64_t)nP, (int)pw,
                        d_observed.get(), d_gram.get(), d_factors.get(), lambda, d_counters.get() + 4);
    });
    FG_CUDA(cudaMemcpyAsync(h_count.get(), d_counters.get() + 4, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    *fallbacks = h_count.get()[0];
    if (*fallbacks == 0 && opt.preconditioner == FG_PRECOND_SCHUR_DIAGONAL && nC) {
      FG_TRY(ensure_cross());
      FG_DISPATCH_WIDTHS(cw, pw, {
        FG_LAUNCH((k_cam_schur_diag<CW_, PW_, TS>), grid_for(nC * 32, 128), 128, 0, st, L, d_cam_edge_off.get(),
                  d_cam_edge.get(), d_edges.get(), d_cross.get(), d_observed.get(), d_gram.get(), d_factors.get(),
                  d_precond.get(), lambda);
      });
    }
    if (*fallbacks == 0 && nC) FG_TRY(write_block_inverses(lambda));
    if (*fallbacks == 0 && nC && learned_blocks) {
      EventTimer ti;
      const bool timed = !learned_compared && opt.learned_policy == 0;  // inference time of the comparison
      if (timed) ti.start(st);
      FG_TRY(ensure_cam_meta());
      const SchurView view = view_at(lambda);
      if (!view.rec) FG_TRY(ensure_cross());
      unsigned nonfinite = 0;
      FG_TRY(gnn_precondition(learned, view, d_minv.get(), st, &nonfinite));
      if (timed) learned_infer_seconds = ti.stop(st);
    }
    if (*fallbacks == 0) FG_TRY(fast.refresh_points(*this, lambda));
    return FG_OK;
  }

  fg_status attach_learned(fg_gnn* g) override {
    if (g) FG_TRY(gnn_check(g, cw, pw, retained / cw, dev));
    learned = g;
    learned_compared = learned_off = false;
    return FG_OK;
  }

  fg_status capture_system(fg_gnn* g, double lambda, size_t probes, uint64_t seed, int kind,
                           size_t* index) override {
    if (kind != 0 && kind != 1) {
      set_error("probe kind must be 0 (products) or 1 (solves)");
      return FG_INVALID_OPTIONS;
    }
    if (!ready || !std::isfinite(lambda) || lambda < 0) {
      set_error("capturing a reduced system requires prepare_damping and a finite nonnegative lambda");
      return FG_INVALID_OPTIONS;
    }
    FG_TRY(gnn_check(g, cw, pw, nC, dev));
    unsigned fb = 0;
    FG_TRY(factor(lambda, &fb));
    if (fb) {
      set_error("local block factorization failed");
      return FG_LINEAR_SOLVE_FAILED;
    }
    FG_TRY(ensure_cross());
    auto apply = [&](const double* x, double* y) -> fg_status {
      PView<double> pv{const_cast<double*>(x), nullptr, nullptr};
      FG_TRY(apply_reduced<double>(pv, lambda, lambda, true, d_tmpd.get(), y, nullptr, nullptr));
      return FG_OK;
    };
    // S^-1 through the block-Jacobi PCG at the backend's tolerance; the work
    // counters and diagnostics of the caller's solves are left untouched
    auto solve = [&](const double* x, double* y) -> fg_status {
      FG_CUDA(cudaMemcpyAsync(d_rhs.get(), x, retained * sizeof(double), cudaMemcpyDeviceToDevice, st));
      const size_t keep_iterations = iterations;
      const fg_schur_diagnostics keep_diag = diag;
      unsigned its = 0;
      int term = FG_TERM_NONE;
      double est = 0;
      size_t ref = 0;
      fg_status s = run_cg(lambda, &its, &term, &est, &ref);
      iterations = keep_iterations;
      diag = keep_diag;
      FG_TRY(s);
      if (term != FG_TERM_CONVERGED) {
        set_error("reduced CG did not converge on a probe");
        return FG_LINEAR_SOLVE_FAILED;
      }
      FG_CUDA(cudaMemcpyAsync(y, d_zred.get(), retained * sizeof(double), cudaMemcpyDeviceToDevice, st));
      return FG_OK;
    };
    FG_TRY(ensure_cam_meta());
    if (kind == 1) return gnn_capture(g, view_at(lambda), probes, seed, 1, solve, d_work.get(), d_qd.get(), st, index);
    return gnn_capture(g, view_at(lambda), probes, seed, 0, apply, d_work.get(), d_qd.get(), st, index);
  }
  // Operator autotuner: times each FP32 single-pass variant that applies to
  // this structure (per-warp TMA rings, direct global loads, prefetching
  // direct loads, TMA-staged stage groups) and keeps the fastest. Runs once
  // per structure shape (device, cameras, points, edges, warp tiles) in the
  // process; the factorization it needs is redone by every solve.
  static constexpr int NVARIANTS = 4;
  struct TunedShape {
    int dev;
    int64_t ncam, npt, nedge, nwt;
    bool operator<(const TunedShape& o) const {
      return std::tie(dev, ncam, npt, nedge, nwt) < std::tie(o.dev, o.ncam, o.npt, o.nedge, o.nwt);
    }
  };
  struct TunedChoice {
    int variant;
    double seconds[NVARIANTS];
  };
  static std::mutex& tuned_mutex() {
    static std::mutex m;
    return m;
  }
  static std::map<TunedShape, TunedChoice>& tuned_shapes() {
    static auto* m = new std::map<TunedShape, TunedChoice>();
    return *m;
  }
  double tuned_seconds[NVARIANTS] = {0, 0, 0, 0};
  fg_status set_poll_limit(unsigned polls) override {
    fast.poll_limit = polls ? polls : RING_POLL_LIMIT;
    drop_graphs();
    return FG_OK;
  }
  void operator_info(int* variant, double* seconds) const override {
    *variant = fast.enabled() ? fast.variant : 0;
    if (seconds)
      for (int v = 0; v < NVARIANTS; ++v) seconds[v] = tuned_seconds[v];
  }
  fg_status autotune_operator() {
    if (!fast.on || !is_f32() || fast.tuned) return FG_OK;
    if (opt.operator_variant >= 1 && opt.operator_variant <= NVARIANTS) {
      fast.variant = fast.variant_ok(opt.operator_variant) ? opt.operator_variant : 1;
      fast.tuned = true;
      drop_graphs();
      return FG_OK;
    }
    const TunedShape shape{dev, (int64_t)nC, (int64_t)nP, (int64_t)nedges, fast.nwt};
    {
      std::lock_guard<std::mutex> lock(tuned_mutex());
      auto it = tuned_shapes().find(shape);
      if (it != tuned_shapes().end()) {
        fast.variant = it->second.variant;
        for (int v = 0; v < NVARIANTS; ++v) tuned_seconds[v] = it->second.seconds[v];
        fast.tuned = true;
        drop_graphs();
        return FG_OK;
      }
    }
    unsigned fb = 0;
    FG_TRY(factor(1.0, &fb));
    if (fb) return FG_OK;
    FG_CUDA(cudaMemsetAsync(d_z.get(), 0, retained * sizeof(TS), st));
    PView<TS> pv{d_z.get(), nullptr, nullptr};
    cudaEvent_t a, b;
    FG_CUDA(cudaEventCreate(&a));
    FG_CUDA(cudaEventCreate(&b));
    float best = 1e30f;
    int best_v = 1;
    for (int v = 1; v <= NVARIANTS; ++v) {
      tuned_seconds[v - 1] = 0;
      if (!fast.variant_ok(v)) continue;
      fast.variant = v;
      FG_TRY(apply_reduced<TS>(pv, 1.0, 1.0, true, d_t.get(), d_q.get(), nullptr, nullptr));
      cudaEventRecord(a, st);
      for (int k = 0; k < 10; ++k)
        FG_TRY(apply_reduced<TS>(pv, 1.0, 1.0, true, d_t.get(), d_q.get(), nullptr, nullptr));
      cudaEventRecord(b, st);
      cudaEventSynchronize(b);
      float ms = 0;
      cudaEventElapsedTime(&ms, a, b);
      tuned_seconds[v - 1] = ms * 1e-3 / 10;
      if (ms < best) {
        best = ms;
        best_v = v;
      }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    fast.variant = best_v;
    fast.tuned = true;
    {
      std::lock_guard<std::mutex> lock(tuned_mutex());
      TunedChoice c{best_v, {}};
      for (int v = 0; v < NVARIANTS; ++v) c.seconds[v] = tuned_seconds[v];
      tuned_shapes()[shape] = c;
    }
    drop_graphs();
    return FG_OK;
  }

  // The reference-layout cross blocks on demand (the fast path skips them).
  fg_status ensure_cross() {
    if (cross_current || !nedges) return FG_OK;
    FG_CUDA(cudaMemsetAsync(d_flags.get() + 1, 0, sizeof(int), st));
    FG_LAUNCH(k_cross<TS>, grid_for(nedges * cw * pw, NT), NT, 0, st, (int64_t)nedges, (int)cw, (int)pw,
              d_edges.get(), d_blocks.get(), d_values.get(), d_scales.get(), d_cross.get(), d_flags.get() + 1);
    cross_current = true;
    return FG_OK;
  }
  const TS* precond_factors() const {
    return opt.preconditioner == FG_PRECOND_SCHUR_DIAGONAL ? d_precond.get() : d_factors.get();
  }

  // out = ax * x + [B x] - E C^-1 E^T x for a double or storage-precision vector.
  template <class TV>
  fg_status apply_reduced(PView<TV> x, double lambda, double ax, bool use_gram, TV* t, TV* out, double* partials,
                          PcgState* pst, const int* gate = nullptr, const double* lam_dev = nullptr) {
    Layout L = layout();
    const int* done = pst ? &pst->done : nullptr;
    if (fast.enabled() && use_gram && ax == lambda)
      return fast.apply(*this, x, lambda, out, partials, pst, gate, lam_dev);
    FG_DISPATCH_WIDTHS(cw, pw, {
      if (nP) FG_LAUNCH((k_points<CW_, PW_, TS, TV>), grid_for(nP, 128), 128, 0, st, L, d_pt_edge_off.get(),
                        d_pt_edge.get(), d_edges.get(), d_cross.get(), d_factors.get(), d_observed.get(), x, lambda, t,
                        done, gate);
      if (nC) FG_LAUNCH((k_cams<CW_, PW_, TS, TV>), grid_for(nC * 32, NT), NT, 0, st, L, d_cam_edge_off.get(),
                        d_cam_edge.get(), d_edges.get(), d_cross.get(), t, d_gram.get(), d_observed.get(), x, ax,
                        (int)use_gram, out, partials, pst, gate);
    });
    return FG_OK;
  }

  // Launch geometry of the wide PCG kernels: whole retained variables per block.
  unsigned wide_block() const { return (unsigned)((256 / cw) * cw); }
  unsigned wide_grid() const {
    size_t per = 256 / cw;
    return grid_for(std::max<size_t>((nC + per - 1) / per, 1), 1);
  }

  // ---- CUDA graph of GRAPH_ITERS PCG iterations on the single-pass operator.
  // Every scalar the iteration needs (alpha, beta, lambda, stopping state)
  // lives in PcgState on the device, so one instantiation serves every solve
  // until buffers are reallocated (prepare / new structure).
  static constexpr int GRAPH_ITERS = 8;
  cudaGraphExec_t g_exec[2] = {nullptr, nullptr};
  uint64_t g_nodes[2] = {0, 0};
  std::vector<uintptr_t> g_key[2];  // what each instantiated graph baked in
  // The whole solve as one graph launch: a WHILE node whose body is
  // COND_ITERS iterations and k_pcg_continue, so the device decides when to
  // stop (no host poll between batches, no gated no-op iterations past
  // convergence beyond the last trip). If the driver refuses the conditional
  // graph, cond_failed switches this backend to the polled graphs above.
  static constexpr int COND_ITERS = 4;
  cudaGraphExec_t c_exec[2] = {nullptr, nullptr};
  uint64_t c_nodes[2] = {0, 0};
  std::vector<uintptr_t> c_key[2];
  bool cond_failed = false;
  void drop_graphs() {
    for (int k = 0; k < 2; ++k) {
      if (g_exec[k]) cudaGraphExecDestroy(g_exec[k]);
      g_exec[k] = nullptr;
      g_key[k].clear();
      if (c_exec[k]) cudaGraphExecDestroy(c_exec[k]);
      c_exec[k] = nullptr;
      c_key[k].clear();
    }
  }
  // Every pointer, size and kernel choice a captured iteration bakes in; a
  // graph whose key no longer matches (a buffer reallocated, another operator
  // variant or coarse state) is re-captured, so a new solve or linearization
  // on the same structure reuses the instantiation.
  std::vector<uintptr_t> graph_key(bool mixed, const double* xd, const PcgState* ps) const {
    return {(uintptr_t)mixed, (uintptr_t)xd, (uintptr_t)ps, (uintptr_t)d_z.get(), (uintptr_t)d_pp.get(),
            (uintptr_t)d_q.get(), (uintptr_t)d_t.get(), (uintptr_t)d_r.get(), (uintptr_t)d_x.get(),
            (uintptr_t)d_partials.get(), (uintptr_t)d_minv.get(), (uintptr_t)d_gram.get(),
            (uintptr_t)d_observed.get(), (uintptr_t)d_tmpd.get(), (uintptr_t)d_qd.get(), (uintptr_t)d_rhs.get(),
            (uintptr_t)d_Wt.get(), (uintptr_t)d_G.get(), (uintptr_t)fast.d_ebeg.get(), (uintptr_t)fast.d_pbeg.get(),
            (uintptr_t)fast.d_erec.get(), (uintptr_t)fast.d_prec.get(), (uintptr_t)fast.d_parts_f.get(),
            (uintptr_t)fast.d_parts_d.get(), (uintptr_t)fast.d_error.get(), (uintptr_t)fast.variant,
            (uintptr_t)fast.d_gacc.get(), (uintptr_t)fast.global_acc, (uintptr_t)fast.poll_limit,
            (uintptr_t)fast.nwt, (uintptr_t)fast.nstages, (uintptr_t)fast.grid, (uintptr_t)coarse_on,
            (uintptr_t)nk, (uintptr_t)nC, (uintptr_t)nP, (uintptr_t)retained, (uintptr_t)dim};
  }
  fg_status iteration_body(bool mixed, double* xd, PcgState* ps, double lambda, int k) {
    double* tsum = d_partials.get() + 4 * 65536;
    PView<TS> pv{d_z.get(), d_pp.get(), &ps->beta};
    FG_TRY(apply_reduced<TS>(pv, lambda, lambda, true, d_t.get(), d_q.get(), tsum, ps, nullptr, &ps->lambda));
    if (!mixed) {
      FG_TRY((launch_update<TS, false>(d_x.get())));
    } else {
      FG_TRY((launch_update<double, true>(xd)));
      if ((k & 3) == 3) FG_TRY(replacement(lambda, xd, ps));
    }
    return FG_OK;
  }
  fg_status launch_continue(cudaGraphConditionalHandle h, bool mixed, PcgState* ps) {
    FG_LAUNCH(k_pcg_continue, 1, 1, 0, st, h, ps, mixed ? 1 : 0, (unsigned)COND_ITERS);
    return FG_OK;
  }
  fg_status capture_cond_graph(bool mixed, double* xd, PcgState* ps, double lambda, cudaGraph_t* out,
                               uint64_t* nodes) {
    FG_CUDA(cudaGraphCreate(out, 0));
    cudaGraphConditionalHandle h;
    FG_CUDA(cudaGraphConditionalHandleCreate(&h, *out, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np = {};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    FG_CUDA(cudaGraphAddNode(&node, *out, nullptr, 0, &np));
    const uint64_t before = g_launches.load();
    FG_CUDA(cudaStreamBeginCaptureToGraph(st, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal));
    fg_status s = FG_OK;
    for (int k = 0; k < COND_ITERS && s == FG_OK; ++k) s = iteration_body(mixed, xd, ps, lambda, k);
    if (s == FG_OK) s = launch_continue(h, mixed, ps);
    cudaGraph_t body = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &body);
    *nodes = g_launches.load() - before;
    g_launches.fetch_sub(*nodes);  // captured, not launched
    FG_TRY(s);
    FG_CUDA(e);
    return FG_OK;
  }
  // Launches the single-launch solve graph (captured on first use per key);
  // the caller reads PcgState back once and adds trips x nodes to the launch
  // count (add_cond_launches).
  fg_status launch_cond_graph(bool mixed, double* xd, PcgState* ps, double lambda) {
    const int g = mixed ? 1 : 0;
    std::vector<uintptr_t> key = graph_key(mixed, xd, ps);
    if (c_exec[g] && key != c_key[g]) {
      cudaGraphExecDestroy(c_exec[g]);
      c_exec[g] = nullptr;
    }
    if (!c_exec[g]) {
      cudaGraph_t graph = nullptr;
      fg_status s = capture_cond_graph(mixed, xd, ps, lambda, &graph, &c_nodes[g]);
      cudaError_t e = s == FG_OK ? cudaGraphInstantiate(&c_exec[g], graph, 0) : cudaSuccess;
      if (graph) cudaGraphDestroy(graph);
      if (s != FG_OK || e != cudaSuccess) {
        c_exec[g] = nullptr;
        cudaGetLastError();
        return s != FG_OK ? s : cuda_status(e, "cudaGraphInstantiate (conditional)");
      }
      c_key[g] = key;
    }
    FG_CUDA(cudaGraphLaunch(c_exec[g], st));
    return FG_OK;
  }
  void add_cond_launches(bool mixed, const PcgState& h) { g_launches.fetch_add((uint64_t)h.trips * c_nodes[mixed]); }

  fg_status launch_graph(bool mixed, double* xd, PcgState* ps, double lambda) {
    const int g = mixed ? 1 : 0;
    std::vector<uintptr_t> key = graph_key(mixed, xd, ps);
    if (g_exec[g] && key != g_key[g]) {
      cudaGraphExecDestroy(g_exec[g]);
      g_exec[g] = nullptr;
    }
    if (!g_exec[g]) {
      g_key[g] = key;
      cudaGraph_t graph = nullptr;
      uint64_t before = g_launches.load();
      FG_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      fg_status s = FG_OK;
      for (int k = 0; k < GRAPH_ITERS && s == FG_OK; ++k) s = iteration_body(mixed, xd, ps, lambda, k);
      cudaError_t e = cudaStreamEndCapture(st, &graph);
      g_nodes[g] = g_launches.load() - before;
      g_launches.fetch_sub(g_nodes[g]);  // captured, not launched
      if (s != FG_OK) {
        if (graph) cudaGraphDestroy(graph);
        return s;
      }
      FG_CUDA(e);
      e = cudaGraphInstantiate(&g_exec[g], graph, 0);
      cudaGraphDestroy(graph);
      if (e != cudaSuccess) {
        g_exec[g] = nullptr;
        return cuda_status(e, "cudaGraphInstantiate");
      }
    }
    FG_CUDA(cudaGraphLaunch(g_exec[g], st));
    g_launches.fetch_add(g_nodes[g]);
    return FG_OK;
  }

  // PCG on S z = b: faer's CG restated (zero start, relative threshold on
  // ||r||_2, callback before the test) with the retained block-Jacobi
  // preconditioner. b is a double retained vector; the solution lands in d_x.
  fg_status pcg(const double* b, double lambda, double rel_tol, size_t max_iters, unsigned* its, int* term,
                double* rel_est) {
    PcgState* ps = d_pcg.get();
    {
      // from the pinned mirror, so the copy is asynchronous; the mirror is
      // rewritten only by the polls below, which the stream orders after it
      PcgState& init = *h_pcg.get();
      init = PcgState{};
      init.max_iterations = (unsigned)std::min<size_t>(max_iters, 0xffffffffu);
      init.lambda = lambda;
      FG_CUDA(cudaMemcpyAsync(ps, &init, sizeof(PcgState), cudaMemcpyHostToDevice, st));
    }
    FG_TRY(launch_start<TS>(b, d_x.get(), rel_tol));
    double* tsum = d_partials.get() + 4 * 65536;
    size_t launched = 0, batch = 4;
    const bool graphed = fast.enabled();
    bool whole = false;  // the single-launch graph ran the solve
    if (graphed && !cond_failed) {
      if (launch_cond_graph(false, nullptr, ps, lambda) == FG_OK) {
        FG_CUDA(cudaMemcpyAsync(h_pcg.get(), ps, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
        FG_CUDA(cudaStreamSynchronize(st));
        add_cond_launches(false, *h_pcg.get());
        whole = true;
      } else {
        cond_failed = true;
      }
    }
    for (bool first = graphed; !whole; first = false) {
      if (!first) {  // the first graph follows the start without a poll (its kernels gate on done)
        FG_CUDA(cudaMemcpyAsync(h_pcg.get(), ps, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
        FG_CUDA(cudaStreamSynchronize(st));
        if (h_pcg.get()->done) break;
      }
      if (launched >= max_iters + 2) break;  // device enforces the limit; host bound is a guard
      if (graphed) {
        FG_TRY(launch_graph(false, nullptr, ps, lambda));
        launched += GRAPH_ITERS;
        continue;
      }
      for (size_t k = 0; k < batch; ++k) {
        PView<TS> pv{d_z.get(), d_pp.get(), &ps->beta};
        FG_TRY(apply_reduced<TS>(pv, lambda, lambda, true, d_t.get(), d_q.get(), tsum, ps));
        FG_TRY((launch_update<TS, false>(d_x.get())));
      }
      launched += batch;
      batch = std::min<size_t>(batch * 2, 64);
    }
    FG_TRY(fast.check(*this));
    const PcgState& h = *h_pcg.get();
    *its = h.iterations;
    *term = h.done ? h.termination : FG_TERM_ITERATION_LIMIT;
    *rel_est = h.bnorm > 0 ? std::sqrt(h.rr) / h.bnorm : 0.0;
    return FG_OK;
  }

  fg_status solve_damped(double lambda, double* predicted, bool copy_to_host) override {
    diag = fg_schur_diagnostics{};
    diag.damping = lambda;
    if (!ready || !std::isfinite(lambda) || lambda < 0) {
      set_error("solve_damped requires prepare_damping and a finite nonnegative lambda");
      return FG_INVALID_OPTIONS;
    }
    solves += 1;
    EventTimer tf, tl, tv;
    if (opt.collect_timings) tf.start(st);
    unsigned fallbacks = 0;
    const bool use_learned = learned_active();
    FG_TRY(factor(lambda, &fallbacks, use_learned));
    if (fallbacks) {  // src/schur.rs:209-215
      if (opt.collect_timings) tim.factorization += tf.stop(st);
      diag.termination = FG_TERM_NOT_POSITIVE_DEFINITE;
      set_error("local block factorization failed");
      return FG_LINEAR_SOLVE_FAILED;
    }
    // scaled_work = -g/D; eliminated part through C^-1; reduced rhs (src/schur.rs:216-242)
    FG_TRY(launch_neg_scaled_gradient());
    FG_TRY(launch_point_solve(lambda));
    FG_TRY(launch_rhs());
    FG_TRY(prepare_coarse(lambda));
    diag.coarse_vectors = coarse_on ? (size_t)nk : 0;
    if (opt.collect_timings) { tim.factorization += tf.stop(st); tl.start(st); }

    unsigned its = 0;
    int term = FG_TERM_NONE;
    double est = 0;
    size_t refinements = 0;
    const bool compare = use_learned && !learned_compared && opt.learned_policy == 0;
    EventTimer tc;
    if (compare) tc.start(st);
    FG_TRY(run_cg(lambda, &its, &term, &est, &refinements));
    if (compare) diag.learned_seconds = learned_infer_seconds + tc.stop(st);
    // a learned preconditioner the comparison switched off runs block-Jacobi
    diag.preconditioner_used = use_learned ? FG_PRECOND_LEARNED
                               : opt.preconditioner == FG_PRECOND_LEARNED ? FG_PRECOND_RETAINED_BLOCKS
                                                                          : opt.preconditioner;
    if (use_learned) {
      // Block-Jacobi stays the yardstick: it takes over when the learned PCG
      // fails, and the first learned solve is compared against it once, on
      // iterations and on device time including the network's inference.
      diag.learned_iterations = its;
      if (term != FG_TERM_CONVERGED || compare) {
        const bool keep = term == FG_TERM_CONVERGED;
        if (keep) {
          FG_TRY(d_keep.resize(std::max<size_t>(retained, 1)));
          FG_CUDA(cudaMemcpyAsync(d_keep.get(), d_zred.get(), retained * sizeof(double), cudaMemcpyDeviceToDevice, st));
        }
        if (compare) tc.start(st);
        FG_TRY(write_block_inverses(lambda));
        unsigned its2 = 0;
        int term2 = FG_TERM_NONE;
        double est2 = 0;
        size_t ref2 = 0;
        FG_TRY(run_cg(lambda, &its2, &term2, &est2, &ref2));
        if (compare) diag.block_jacobi_seconds = tc.stop(st);
        diag.block_jacobi_iterations = its2;
        if (!keep) {
          diag.learned_fallback = 1;
        } else {
          learned_compared = true;
          if (term2 == FG_TERM_CONVERGED && (its2 < its || diag.block_jacobi_seconds < diag.learned_seconds)) {
            learned_off = true;
            diag.learned_fallback = 2;
          } else {
            FG_CUDA(cudaMemcpyAsync(d_zred.get(), d_keep.get(), retained * sizeof(double), cudaMemcpyDeviceToDevice,
                                    st));
            final_residual_known = false;  // h_pcg describes the block-Jacobi solve
            term2 = term;
            est2 = est;
            ref2 = refinements;
          }
        }
        if (diag.learned_fallback) diag.preconditioner_used = FG_PRECOND_RETAINED_BLOCKS;
        term = term2;
        est = est2;
        refinements += ref2;
        its += its2;
        diag.iterations = its;
      }
    }
    diag.termination = term;
    diag.refinements = refinements;
    if (term == FG_TERM_CONVERGED) {
      diag.estimated_relative_residual = est;
      diag.has_estimated = 1;
    }
    if (opt.collect_timings) { tim.linear_solve += tl.stop(st); tv.start(st); }
    // recover step (src/schur.rs:312-344) and verify (src/schur.rs:346-397)
    FG_TRY(launch_recover(lambda));
    double pred = 0;
    fg_status vs = verify(lambda, &pred);
    if (opt.collect_timings) tim.verification += tv.stop(st);
    if (vs != FG_OK) return vs;
    if (copy_to_host) {
      FG_CUDA(cudaMemcpyAsync(h_step.get(), d_step.get(), dim * sizeof(double), cudaMemcpyDeviceToHost, st));
      FG_CUDA(cudaStreamSynchronize(st));
    }
    if (diag.termination != FG_TERM_CONVERGED) {
      set_error("reduced CG did not converge");
      return FG_LINEAR_SOLVE_FAILED;
    }
    *predicted = pred;
    return FG_OK;
  }

  // One reduced solve with the inverses currently in d_minv; the solution
  // lands in d_zred (f64).
  fg_status run_cg(double lambda, unsigned* its, int* term, double* est, size_t* refinements) {
    final_residual_known = false;
    if (std::is_same<TS, double>::value) {
      FG_TRY(pcg(d_rhs.get(), lambda, opt.relative_tolerance, opt.max_iterations, its, term, est));
      FG_TRY(launch_widen(d_x.get(), d_zred.get(), retained));
      iterations += *its;
      diag.iterations = *its;
      return FG_OK;
    }
    return refine(lambda, its, term, est, refinements);
  }

  // FP32 PCG with FP64 residual replacement (reliable updates): the Krylov
  // recurrences run in the storage precision while the iterate accumulates in
  // FP64; whenever the recurrence residual has fallen by residual_replacement
  // (and before declaring convergence) it is replaced by b - S x evaluated in
  // FP64 arithmetic. Convergence is only ever declared on that FP64 residual.
  fg_status refine(double lambda, unsigned* its_out, int* term_out, double* est_out, size_t* rounds) {
    PcgState* ps = d_pcg.get();
    double* xd = d_zred.get();
    {
      PcgState& init = *h_pcg.get();  // pinned mirror: asynchronous copy (see pcg())
      init = PcgState{};
      init.max_iterations = (unsigned)std::min<size_t>(opt.max_iterations, 0xffffffffu);
      init.lambda = lambda;
      const double d = replacement_factor();
      init.delta2 = d * d;
      FG_CUDA(cudaMemcpyAsync(ps, &init, sizeof(PcgState), cudaMemcpyHostToDevice, st));
    }
    FG_TRY(launch_start<double>(d_rhs.get(), xd, opt.relative_tolerance));
    double* tsum = d_partials.get() + 4 * 65536;
    size_t launched = 0, batch = 4;
    const size_t max_iters = opt.max_iterations;
    const bool graphed = fast.enabled();
    bool whole = false;  // the single-launch graph ran the solve
    if (graphed && !cond_failed) {
      if (launch_cond_graph(true, xd, ps, lambda) == FG_OK) {
        FG_CUDA(cudaMemcpyAsync(h_pcg.get(), ps, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
        FG_CUDA(cudaStreamSynchronize(st));
        add_cond_launches(true, *h_pcg.get());
        whole = true;
      } else {
        cond_failed = true;
      }
    }
    for (bool first = graphed; !whole; first = false) {
      if (!first) {  // the first graph follows the start without a poll
        FG_CUDA(cudaMemcpyAsync(h_pcg.get(), ps, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
        FG_CUDA(cudaStreamSynchronize(st));
        if (h_pcg.get()->done == 1) break;
      }
      if (launched >= max_iters + 8) break;  // guard; the device enforces the limit
      if (graphed) {
        FG_TRY(launch_graph(true, xd, ps, lambda));
        launched += GRAPH_ITERS;
        continue;
      }
      for (size_t k = 0; k < batch; ++k) {
        PView<TS> pv{d_z.get(), d_pp.get(), &ps->beta};
        FG_TRY(apply_reduced<TS>(pv, lambda, lambda, true, d_t.get(), d_q.get(), tsum, ps));
        FG_TRY((launch_update<double, true>(xd)));
        if ((k & 3) == 3) FG_TRY(replacement(lambda, xd, ps));
      }
      launched += batch;
      batch = std::min<size_t>(batch * 2, 64);
    }
    FG_TRY(fast.check(*this));
    const PcgState& h = *h_pcg.get();
    iterations += h.iterations;
    diag.iterations = h.iterations;
    *its_out = h.iterations;
    *term_out = h.done == 1 ? h.termination : FG_TERM_ITERATION_LIMIT;
    *est_out = h.bnorm > 0 ? std::sqrt(h.rr_last) / h.bnorm : 0.0;
    *rounds = h.replacements;
    final_residual_known = h.done == 1 && h.termination == FG_TERM_CONVERGED;
    return FG_OK;
  }

  // Spacing of the FP64 residual replacements: the requested factor, or the
  // reduction from ||b|| to the relative tolerance split into the fewest equal
  // factors of at most 1e-4 (four decades per FP32 stretch). Longer stretches
  // let the FP32 recurrence drift far enough to delay convergence by tens of
  // iterations at tolerances far below FP32 precision; shorter ones cost
  // replacements.
  double replacement_factor() const {
    const double r = opt.residual_replacement;
    if (r > 0 && r < 1) return r;
    const double tol = opt.relative_tolerance > 0 && opt.relative_tolerance < 1 ? opt.relative_tolerance : 1e-10;
    const double decades = -std::log10(tol);
    const double stretches = std::max(1.0, std::ceil(decades / 4.0 - 1e-9));
    return std::pow(tol, 1.0 / stretches);
  }

  // Gated FP64 residual replacement: runs only while the device flag is set.
  fg_status replacement(double lambda, double* xd, PcgState* ps) {
    PView<double> xv{xd, nullptr, nullptr};
    FG_TRY(apply_reduced<double>(xv, lambda, lambda, true, d_tmpd.get(), d_qd.get(), nullptr, nullptr, &ps->replace,
                                 &ps->lambda));
    return launch_replace();
  }

  // ---- kernels launched by solve_damped (defined below as members)
  fg_status launch_neg_scaled_gradient();
  fg_status launch_point_solve(double lambda);
  fg_status launch_rhs();
  fg_status launch_widen(const TS* x, double* out, size_t n);
  fg_status launch_axpy_widen(const TS* x, double* out, size_t n);
  fg_status launch_recover(double lambda);
  fg_status verify(double lambda, double* predicted);
  fg_status device_dot(const double* a, const double* b, size_t n, double* out);
  fg_status reduced_residual_d(double lambda, const double* z, double* res, double* rnorm);

  // ------------------------------------------------------------- accessors
  fg_status step_norm_inf(double* out) override { return device_norm_inf(d_step.get(), dim, out); }
  fg_status step_norm_async(double* d_out) override {
    if (dim == 0) {
      FG_CUDA(cudaMemsetAsync(d_out, 0, 2 * sizeof(double), st));
      return FG_OK;
    }
    unsigned g = std::min<unsigned>(grid_for(dim, NT), 4 * nsm);
    FG_LAUNCH(k_norm_inf<double>, g, NT, 0, st, (int64_t)dim, (const double*)d_step.get(), d_partials.get(),
              d_counters.get() + 3, d_out);
    return FG_OK;
  }
  const double* step_host() const override { return h_step.get(); }
  const double* step_device() const override { return d_step.get(); }
  size_t dimension() const override { return dim; }
  void work(size_t* s, size_t* i) const override { *s = solves; *i = iterations; }
  void diagnostics(fg_schur_diagnostics* d) const override { *d = diag; }
  void timings(fg_schur_timings* t) const override { *t = tim; }
  bool is_f32() const override { return !std::is_same<TS, double>::value; }
  int device() const override { return dev; }
  cudaStream_t stream() const override { return st; }
  void* values_device() override { return d_values.get(); }
  double* negres_device() override { return d_negres.get(); }
  void mark_device_model(size_t nrows) override {
    source = DEVICE_BAL;
    rows = nrows;
    device_model_current = true;
    gradient_current = false;
    ready = false;
  }

  fg_status bind_bal(const BalObservations& ob) override {
    const uint64_t id = ob.problem_id;
    const size_t cams = ob.cameras, pts = ob.points, obs = ob.observations;
    if (cw != 9 || pw != 3) return FG_UNSUPPORTED_STRUCTURE;
    if (retained != 9 * cams || dim != 9 * cams + 3 * pts) return FG_DIMENSION_MISMATCH;
    if (bal_bound == id && structure_valid) return FG_OK;
    FG_TRY(build_structure_bal(cams, pts, obs, ob.cam, ob.pt));
    up_blocks.clear();
    up_edges.clear();
    nvalues = 24 * obs;
    FG_TRY(d_values.resize(std::max<size_t>(nvalues, 1)));
    FG_TRY(d_negres.resize(std::max<size_t>(2 * obs, 1)));
    bal_bound = id;
    bal_obs = obs;
    return FG_OK;
  }

  fg_status structure_sizes(size_t* nb, size_t* ne, size_t* nv, size_t* nvar, size_t* r, size_t* c) override {
    FG_TRY(sync_model());
    size_t vars = 0;
    for (uint8_t o : h_observed) vars += o;
    if (nb) *nb = nblocks;
    if (ne) *ne = nedges;
    if (nv) *nv = nvalues;
    if (nvar) *nvar = vars;
    if (r) *r = rows;
    if (c) *c = dim;
    return FG_OK;
  }

  fg_status model_host(HostModel* m) override {
    size_t nb = 0, nv = 0, r = 0, c = 0;
    FG_TRY(structure_sizes(&nb, nullptr, &nv, nullptr, &r, &c));
    std::vector<uint64_t> b5(5 * std::max<size_t>(nb, 1));
    FG_TRY(export_structure(b5.data(), nullptr, nullptr, nullptr));
    m->rows = r;
    m->cols = c;
    m->values.assign(std::max<size_t>(nv, 1), 0.0);
    m->negres.assign(std::max<size_t>(r, 1), 0.0);
    FG_TRY(export_model(m->values.data(), m->negres.data(), nullptr, nullptr, nullptr, nullptr));
    m->blocks.resize(nb);
    for (size_t i = 0; i < nb; ++i)
      m->blocks[i] = HostBlock{b5[5 * i], b5[5 * i + 1], b5[5 * i + 2], b5[5 * i + 3], b5[5 * i + 4]};
    return FG_OK;
  }

  fg_status export_structure(uint64_t* b5, uint64_t* e4, uint64_t* owners, uint64_t* v3) override {
    FG_TRY(sync_model());
    std::vector<DBlockMeta> mb(nblocks);
    std::vector<DEdgeMeta> me(nedges);
    if (nblocks) FG_CUDA(cudaMemcpy(mb.data(), d_blocks.get(), nblocks * sizeof(DBlockMeta), cudaMemcpyDeviceToHost));
    if (nedges) FG_CUDA(cudaMemcpy(me.data(), d_edges.get(), nedges * sizeof(DEdgeMeta), cudaMemcpyDeviceToHost));
    if (b5)
      for (size_t i = 0; i < nblocks; ++i) {
        b5[5 * i] = mb[i].row; b5[5 * i + 1] = mb[i].col; b5[5 * i + 2] = mb[i].rows;
        b5[5 * i + 3] = mb[i].cols; b5[5 * i + 4] = mb[i].start;
      }
    if (e4)
      for (size_t e = 0; e < nedges; ++e) {
        e4[4 * e] = (uint64_t)me[e].cam * cw; e4[4 * e + 1] = (uint64_t)me[e].pt * pw;
        e4[4 * e + 2] = me[e].lblk; e4[4 * e + 3] = me[e].rblk;
      }
    // First-appearance variable ids (block_factors.rs:52-87).
    std::vector<uint64_t> own(dim, UINT64_MAX);
    std::vector<uint64_t> vars;
    for (size_t i = 0; i < nblocks; ++i) {
      if (mb[i].cols == 0) continue;
      size_t col = mb[i].col;
      if (own[col] == UINT64_MAX) {
        uint64_t id = vars.size() / 3;
        size_t gstart = vars.empty() ? 0 : vars[vars.size() - 1] + vars[vars.size() - 2] * vars[vars.size() - 2];
        vars.push_back(col); vars.push_back(mb[i].cols); vars.push_back(gstart);
        for (size_t c = col; c < col + mb[i].cols; ++c) own[c] = id;
      }
    }
    if (owners) std::copy(own.begin(), own.end(), owners);
    if (v3) std::copy(vars.begin(), vars.end(), v3);
    return FG_OK;
  }

  fg_status export_model(double* values, double* negres, double* g, double* scales, double* gram,
                         double* cross) override {
    FG_TRY(sync_model());
    FG_CUDA(cudaStreamSynchronize(st));
    auto fetch = [&](const TS* src, size_t n, double* dst) -> fg_status {
      if (!dst || !n) return FG_OK;
      std::vector<TS> tmp(n);
      FG_CUDA(cudaMemcpy(tmp.data(), src, n * sizeof(TS), cudaMemcpyDeviceToHost));
      for (size_t i = 0; i < n; ++i) dst[i] = (double)tmp[i];
      return FG_OK;
    };
    FG_TRY(fetch(d_values.get(), nvalues, values));
    if (negres && rows) FG_CUDA(cudaMemcpy(negres, d_negres.get(), rows * sizeof(double), cudaMemcpyDeviceToHost));
    if (g && dim) FG_CUDA(cudaMemcpy(g, d_g.get(), dim * sizeof(double), cudaMemcpyDeviceToHost));
    if (scales && dim && ready) FG_CUDA(cudaMemcpy(scales, d_scales.get(), dim * sizeof(double), cudaMemcpyDeviceToHost));
    if (gram && ready) {
      // first-appearance order, packed w*w per variable
      std::vector<uint64_t> v3;
      size_t nvar = 0;
      for (uint8_t o : h_observed) nvar += o;
      v3.resize(3 * nvar);
      FG_TRY(export_structure(nullptr, nullptr, nullptr, v3.data()));
      size_t ng = nC * cw * cw + nP * pw * pw;
      std::vector<double> all(ng);
      FG_TRY(fetch(d_gram.get(), ng, all.data()));
      for (size_t i = 0; i < nvar; ++i) {
        size_t col = v3[3 * i], w = v3[3 * i + 1], start = v3[3 * i + 2];
        size_t go = col < retained ? (col / cw) * cw * cw : nC * cw * cw + ((col - retained) / pw) * pw * pw;
        for (size_t k = 0; k < w * w; ++k) gram[start + k] = all[go + k];
      }
    }
    if (cross && ready) {
      FG_TRY(ensure_cross());
      FG_CUDA(cudaStreamSynchronize(st));
      FG_TRY(fetch(d_cross.get(), nedges * cw * pw, cross));
    }
    return FG_OK;
  }

  fg_status time_operator(double lambda, size_t reps, double* seconds, double* bytes) override {
    if (!ready) return FG_INVALID_OPTIONS;
    unsigned fb = 0;
    FG_TRY(factor(lambda, &fb));
    FG_CUDA(cudaMemsetAsync(d_z.get(), 0, retained * sizeof(TS), st));
    PView<TS> pv{d_z.get(), nullptr, nullptr};
    FG_TRY(apply_reduced<TS>(pv, lambda, lambda, true, d_t.get(), d_q.get(), nullptr, nullptr));  // warm
    cudaEvent_t a, b;
    FG_CUDA(cudaEventCreate(&a));
    FG_CUDA(cudaEventCreate(&b));
    FG_CUDA(cudaEventRecord(a, st));
    for (size_t k = 0; k < reps; ++k) FG_TRY(apply_reduced<TS>(pv, lambda, lambda, true, d_t.get(), d_q.get(), nullptr, nullptr));
    FG_CUDA(cudaEventRecord(b, st));
    FG_CUDA(cudaEventSynchronize(b));
    FG_TRY(fast.check(*this));
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *seconds = reps ? ms * 1e-3 / (double)reps : 0.0;
    double s = (double)sizeof(TS);
    // cross blocks + edge index, point factor (lower) + edge offset, camera Gram (lower) + x + y
    *bytes = (double)nedges * (cw * pw * s + 4.0) + (double)nP * (pw * (pw + 1) / 2 * s + 4.0) +
             (double)nC * (cw * (cw + 1) / 2 * s + 2.0 * cw * s);
    return FG_OK;
  }

  fg_status time_operator_kernel(double lambda, size_t reps, double* seconds, double* bytes) override {
    if (!ready) return FG_INVALID_OPTIONS;
    if (!fast.enabled()) return FG_UNSUPPORTED_STRUCTURE;
    unsigned fb = 0;
    FG_TRY(factor(lambda, &fb));
    FG_CUDA(cudaMemsetAsync(d_z.get(), 0, retained * sizeof(TS), st));
    PView<TS> pv{d_z.get(), nullptr, nullptr};
    FG_TRY(fast.apply(*this, pv, lambda, d_q.get(), nullptr, nullptr, nullptr, nullptr, false));  // warm
    cudaEvent_t a, b;
    FG_CUDA(cudaEventCreate(&a));
    FG_CUDA(cudaEventCreate(&b));
    FG_CUDA(cudaEventRecord(a, st));
    for (size_t k = 0; k < reps; ++k)
      FG_TRY(fast.apply(*this, pv, lambda, d_q.get(), nullptr, nullptr, nullptr, nullptr, false));
    FG_CUDA(cudaEventRecord(b, st));
    FG_CUDA(cudaEventSynchronize(b));
    FG_TRY(fast.settle(*this));
    FG_TRY(fast.check(*this));
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *seconds = reps ? ms * 1e-3 / (double)reps : 0.0;
    const double s = (double)sizeof(TS);
    // cross blocks + edge index, point factor (lower) + edge offset, x in, camera sums out
    *bytes = (double)nedges * (cw * pw * s + 4.0) + (double)nP * (pw * (pw + 1) / 2 * s + 4.0) +
             (double)nC * (2.0 * cw * s);
    return FG_OK;
  }

  fg_status reduced_apply(double lambda, const double* x, double* y) override {
    if (!ready) return FG_INVALID_OPTIONS;
    unsigned fb = 0;
    FG_TRY(factor(lambda, &fb));
    FG_CUDA(cudaMemcpyAsync(d_work.get(), x, retained * sizeof(double), cudaMemcpyHostToDevice, st));
    PView<double> pv{d_work.get(), nullptr, nullptr};
    FG_TRY(apply_reduced<double>(pv, lambda, lambda, true, d_tmpd.get(), d_qd.get(), nullptr, nullptr));
    FG_CUDA(cudaMemcpyAsync(y, d_qd.get(), retained * sizeof(double), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    return FG_OK;
  }
};

}  // namespace fg

#include "schur_solve.cuh"

namespace fg {

fg_status make_schur(size_t retained, size_t cw, size_t pw, const fg_schur_options& o, Backend** out) {
  if (cw > (size_t)MAXW || pw > (size_t)MAXW) {
    set_error("block widths above 16 are not supported");
    return FG_INVALID_OPTIONS;
  }
  if (o.precision == FG_PRECISION_F32_REFINED) {
    auto* b = new SchurImpl<float>(retained, cw, pw, o);
    fg_status s = b->init();
    if (s != FG_OK) { delete b; return s; }
    *out = b;
  } else if (o.precision == FG_PRECISION_F64) {
    auto* b = new SchurImpl<double>(retained, cw, pw, o);
    fg_status s = b->init();
    if (s != FG_OK) { delete b; return s; }
    *out = b;
  } else {
    set_error("unknown precision");
    return FG_INVALID_OPTIONS;
  }
  return FG_OK;
}

}  // namespace fg
