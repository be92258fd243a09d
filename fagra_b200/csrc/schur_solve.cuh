// Right-hand side, back-substitution and verification of one damped Schur
// attempt (src/schur.rs:204-247, 312-397; src/linear_model.rs:233-282).
#pragma once

namespace fg {

static __global__ void k_neg_scaled_gradient(int64_t n, const double* g, const double* d, double* out) {
  int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < n) out[j] = -g[j] / d[j];
}

// In place w_p = C_p^-1 w_p for every eliminated variable (block_factors.rs:178-204).
template <int PW, class TS>
static __global__ void k_point_solve(Layout L, const TS* factors, const uint8_t* observed, double* w, double lambda) {
  int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (pt >= L.nP) return;
  const int pw = PW ? PW : L.pw;
  constexpr int PM = PW ? PW : MAXW;
  double v[PM];
  double* base = w + L.retained + pt * pw;
  for (int p = 0; p < pw; ++p) v[p] = base[p];
  int64_t var = L.nC + pt;
  if (observed[var]) llt_solve<PW, TS, double>(factors + L.gram_offset(var), v, pw);
  else if (lambda != 0) for (int p = 0; p < pw; ++p) v[p] /= lambda;
  for (int p = 0; p < pw; ++p) base[p] = v[p];
}

template <class TS>
static __global__ void k_widen(int64_t n, const TS* x, double* out, int accumulate) {
  int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < n) out[j] = accumulate ? out[j] + (double)x[j] : (double)x[j];
}

// z_p = C_p^-1 (-g_p/D_p - sum_e E_e^T z_c); step = z / D (src/schur.rs:312-344).
template <int CW, int PW, class TS>
static __global__ void k_recover_points(Layout L, const int64_t* pt_edge_off, const int64_t* pt_edge, const DEdgeMeta* edges,
                                 const TS* cross, const TS* factors, const uint8_t* observed, const double* g,
                                 const double* scales, const double* zred, double lambda, double* step) {
  int64_t pt = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (pt >= L.nP) return;
  const int cw = CW ? CW : L.cw, pw = PW ? PW : L.pw;
  constexpr int PM = PW ? PW : MAXW;
  double acc[PM];
  int64_t base = L.retained + pt * pw;
  for (int p = 0; p < pw; ++p) acc[p] = -g[base + p] / scales[base + p];
  for (int64_t k = pt_edge_off[pt]; k < pt_edge_off[pt + 1]; ++k) {
    int64_t e = pt_edge[k];
    int64_t cam = edges[e].cam;
    const TS* E = cross + e * (int64_t)cw * pw;
    for (int p = 0; p < pw; ++p) {
      double s = 0;
      for (int c = 0; c < cw; ++c) s += (double)E[p * cw + c] * zred[cam * cw + c];
      acc[p] -= s;
    }
  }
  int64_t var = L.nC + pt;
  if (observed[var]) llt_solve<PW, TS, double>(factors + L.gram_offset(var), acc, pw);
  else if (lambda != 0) for (int p = 0; p < pw; ++p) acc[p] /= lambda;
  for (int p = 0; p < pw; ++p) step[base + p] = acc[p] / scales[base + p];
}

static __global__ void k_step_cams(int64_t n, const double* zred, const double* scales, double* step) {
  int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (j < n) step[j] = zred[j] / scales[j];
}

// jd = J delta per emission (src/linear_model.rs:39-55); partial ||J delta||^2.
template <class TS>
static __global__ void k_jdelta(int64_t nemi, const int64_t* emi_off, const DBlockMeta* blocks, const TS* values,
                         const double* delta, double* jd, double* partials, VerifyState* vs) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double s2 = 0;
  if (e < nemi) {
    int64_t b0 = emi_off[e], b1 = emi_off[e + 1];
    if (b1 > b0) {
      DBlockMeta f = blocks[b0];
      for (int i = 0; i < f.rows; ++i) {
        double y = 0;
        for (int64_t b = b0; b < b1; ++b) {
          DBlockMeta m = blocks[b];
          const TS* v = values + m.start + i;
          for (int j = 0; j < m.cols; ++j) y += (double)v[(int64_t)j * m.rows] * delta[m.col + j];
        }
        jd[f.row + i] = y;
        s2 += y * y;
      }
    }
  }
  double v[1] = {s2};
  block_sums<1>(v);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
  if (arrive_last(&vs->counter0)) {
    double tot[1];
    finish_sums<1>(partials, tot);
    if (threadIdx.x == 0) {
      vs->jd2 = tot[0];
      vs->counter0 = 0;
    }
  }
}

// J delta for the device BAL layout (one emission per observation: rows 2k and
// 2k+1, values [24k, 24k+24) = camera 2x9 then point 2x3, column major) with
// 16-byte loads of each emission's values; same sums as k_jdelta. Grid-stride
// over the emissions with a grid of a few blocks per SM, so the last block
// sums only a few hundred partials.
template <class TS>
static __global__ void k_jdelta_bal(int64_t nobs, int64_t retained, const DEdgeMeta* edges, const TS* values,
                                    const double* delta, double* jd, double* partials, VerifyState* vs) {
  double s2 = 0;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nobs; k += (int64_t)gridDim.x * blockDim.x) {
    double v[18], w[6];
    bal_cam_block<TS>(values, k, v);
    bal_pt_block<TS>(values, k, w);
    const int2 cp = *reinterpret_cast<const int2*>(edges + k);  // (camera, point)
    const double* dc = delta + 9 * (int64_t)cp.x;
    const double* dp = delta + retained + 3 * (int64_t)cp.y;
    double y0 = 0, y1 = 0;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      const double d = dc[c];
      y0 += v[2 * c] * d;
      y1 += v[2 * c + 1] * d;
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double d = dp[c];
      y0 += w[2 * c] * d;
      y1 += w[2 * c + 1] * d;
    }
    *reinterpret_cast<double2*>(jd + 2 * k) = make_double2(y0, y1);
    s2 += y0 * y0 + y1 * y1;
  }
  double w[1] = {s2};
  block_sums<1>(w);
  if (threadIdx.x == 0) partials[blockIdx.x] = w[0];
  if (arrive_last(&vs->counter0)) {
    double tot[1];
    finish_sums<1>(partials, tot);
    if (threadIdx.x == 0) {
      vs->jd2 = tot[0];
      vs->counter0 = 0;
    }
  }
}

// Full damped normal residual J^T (J delta + r) + lambda D^2 delta per
// coordinate (src/linear_model.rs:254-281) with every norm the diagnostics need.
template <class TS>
static __global__ void k_normal_residual(Layout L, const int64_t* var_off, const int64_t* var_blk, const DBlockMeta* blocks,
                                  const TS* values, const double* jd, const double* negres, const double* g,
                                  const double* scales, const double* delta, double lambda, const double* camjt,
                                  double* partials, VerifyState* vs, const int64_t* bal_pt_off,
                                  const int64_t* bal_pt_edge) {
  double acc[6] = {0, 0, 0, 0, 0, 0};
  auto add = [&](double nr, int64_t j) {  // the per-coordinate terms of the diagnostics
    const double s = scales[j], d = delta[j];
    nr += (lambda * (s * d)) * s;
    const double gj = g[j];
    acc[0] += nr * nr;
    acc[1] += gj * gj;
    acc[2] += (nr / s) * (nr / s);
    acc[3] += (gj / s) * (gj / s);
    acc[4] += gj * d;
    acc[5] += isfinite(d) ? 0.0 : 1.0;
  };
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (bal_pt_off && camjt) {
    // device BAL layout: camera coordinates from camjt, then one thread per
    // point walks its emissions once for its 3 coordinates
    for (int64_t j = t0; j < L.retained; j += stride) add(camjt[j], j);
    for (int64_t pt = t0; pt < L.nP; pt += stride) {
      double n0 = 0, n1 = 0, n2 = 0;
      for (int64_t k = bal_pt_off[pt]; k < bal_pt_off[pt + 1]; ++k) {
        const int64_t e = bal_pt_edge[k];
        double w[6];
        bal_pt_block<TS>(values, e, w);
        const double2 jj = *reinterpret_cast<const double2*>(jd + 2 * e);
        const double2 nn = *reinterpret_cast<const double2*>(negres + 2 * e);
        const double r0 = jj.x - nn.x, r1 = jj.y - nn.y;
        n0 += w[0] * r0 + w[1] * r1;
        n1 += w[2] * r0 + w[3] * r1;
        n2 += w[4] * r0 + w[5] * r1;
      }
      const int64_t j = L.retained + 3 * pt;
      add(n0, j);
      add(n1, j + 1);
      add(n2, j + 2);
    }
  }
  for (int64_t j = t0; !(bal_pt_off && camjt) && j < L.dim; j += stride) {
    int64_t v;
    int off;
    L.locate(j, &v, &off);
    double nr = 0;
    if (camjt && j < L.retained) {
      nr = camjt[j];
    } else if (bal_pt_off) {  // device BAL layout: the point's emissions, 2 rows each
      const int64_t pt = v - L.nC;
      for (int64_t k = bal_pt_off[pt]; k < bal_pt_off[pt + 1]; ++k) {
        const int64_t e = bal_pt_edge[k];
        const TS* col = values + 24 * e + 18 + 2 * off;
        nr += (double)col[0] * (jd[2 * e] - negres[2 * e]) + (double)col[1] * (jd[2 * e + 1] - negres[2 * e + 1]);
      }
    } else for (int64_t k = var_off[v]; k < var_off[v + 1]; ++k) {
      DBlockMeta b = blocks[var_blk[k]];
      const TS* col = values + b.start + (int64_t)off * b.rows;
      double s = 0;
      for (int i = 0; i < b.rows; ++i) s += (double)col[i] * (jd[b.row + i] - negres[b.row + i]);
      nr += s;
    }
    add(nr, j);
  }
  block_sums<6>(acc);
  if (threadIdx.x == 0)
    for (int k = 0; k < 6; ++k) partials[6 * blockIdx.x + k] = acc[k];
  if (arrive_last(&vs->counter1)) {
    double tot[6];
    finish_sums<6>(partials, tot);
    if (threadIdx.x == 0) {
      vs->nr2 = tot[0];
      vs->g2 = tot[1];
      vs->snr2 = tot[2];
      vs->sg2 = tot[3];
      vs->gd = tot[4];
      vs->nonfinite_step = tot[5] != 0;
      vs->counter1 = 0;
    }
  }
}

// res = rhs - q (or q - rhs with sign -1); sums ||res||^2 and ||rhs||^2 into out2.
static __global__ void k_sub_norms(int64_t n, const double* q, const double* rhs, double sign, double* res, double* partials,
                            unsigned* counter, double* out2) {
  double a = 0, b = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double r = sign * (rhs[i] - q[i]);
    if (res) res[i] = r;
    a += r * r;
    b += rhs[i] * rhs[i];
  }
  double v[2] = {a, b};
  block_sums<2>(v);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = v[0];
    partials[2 * blockIdx.x + 1] = v[1];
  }
  if (arrive_last(counter)) {
    double tot[2];
    finish_sums<2>(partials, tot);
    if (threadIdx.x == 0) {
      out2[0] = tot[0];
      out2[1] = tot[1];
      *counter = 0;
    }
  }
}

static __global__ void k_dot(int64_t n, const double* a, const double* b, double* partials, unsigned* counter, double* out) {
  double s = 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += a[i] * b[i];
  double v[1] = {s};
  block_sums<1>(v);
  if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
  if (arrive_last(counter)) {
    double tot[1];
    finish_sums<1>(partials, tot);
    if (threadIdx.x == 0) {
      out[0] = tot[0];
      *counter = 0;
    }
  }
}

template <class TS>
fg_status SchurImpl<TS>::launch_neg_scaled_gradient() {
  if (dim) FG_LAUNCH(k_neg_scaled_gradient, grid_for(dim, NT), NT, 0, st, (int64_t)dim, d_g.get(), d_scales.get(),
                     d_work.get());
  return FG_OK;
}

template <class TS>
fg_status SchurImpl<TS>::launch_point_solve(double lambda) {
  if (!nP) return FG_OK;
  Layout L = layout();
  FG_DISPATCH_WIDTHS(cw, pw, {
    FG_LAUNCH((k_point_solve<PW_, TS>), grid_for(nP, 128), 128, 0, st, L, d_factors.get(), d_observed.get(),
              d_work.get(), lambda);
  });
  return FG_OK;
}

template <class TS>
fg_status SchurImpl<TS>::launch_rhs() {
  if (!nC) return FG_OK;
  if (fast.enabled() && !cross_current) return fast.rhs(*this, d_work.get(), d_rhs.get());
  Layout L = layout();
  PView<double> w{d_work.get(), nullptr, nullptr};
  FG_DISPATCH_WIDTHS(cw, pw, {
    FG_LAUNCH((k_cams<CW_, PW_, TS, double>), grid_for(nC * 32, NT), NT, 0, st, L, d_cam_edge_off.get(),
              d_cam_edge.get(), d_edges.get(), d_cross.get(), d_work.get() + retained, d_gram.get(),
              d_observed.get(), w, 1.0, 0, d_rhs.get(), (double*)nullptr, (PcgState*)nullptr, (const int*)nullptr);
  });
  return FG_OK;
}

template <class TS>
fg_status SchurImpl<TS>::launch_widen(const TS* x, double* out, size_t n) {
  if (n) FG_LAUNCH(k_widen<TS>, grid_for(n, NT), NT, 0, st, (int64_t)n, x, out, 0);
  return FG_OK;
}
template <class TS>
fg_status SchurImpl<TS>::launch_axpy_widen(const TS* x, double* out, size_t n) {
  if (n) FG_LAUNCH(k_widen<TS>, grid_for(n, NT), NT, 0, st, (int64_t)n, x, out, 1);
  return FG_OK;
}

template <class TS>
fg_status SchurImpl<TS>::launch_recover(double lambda) {
  Layout L = layout();
  if (retained) FG_LAUNCH(k_step_cams, grid_for(retained, NT), NT, 0, st, (int64_t)retained, d_zred.get(),
                          d_scales.get(), d_step.get());
  if (nP && fast.enabled() && !cross_current) {
    FG_CUDA(cudaMemsetAsync(d_step.get() + retained, 0, (dim - retained) * sizeof(double), st));
    return fast.recover(*this, d_zred.get(), d_g.get(), d_scales.get(), d_step.get());
  }
  if (nP) {
    FG_DISPATCH_WIDTHS(cw, pw, {
      FG_LAUNCH((k_recover_points<CW_, PW_, TS>), grid_for(nP, 128), 128, 0, st, L, d_pt_edge_off.get(),
                d_pt_edge.get(), d_edges.get(), d_cross.get(), d_factors.get(), d_observed.get(), d_g.get(),
                d_scales.get(), d_zred.get(), lambda, d_step.get());
    });
  }
  return FG_OK;
}

template <class TS>
fg_status SchurImpl<TS>::device_dot(const double* a, const double* b, size_t n, double* out) {
  if (!n) { *out = 0; return FG_OK; }
  unsigned g = std::min<unsigned>(grid_for(n, NT), 4 * nsm);
  FG_LAUNCH(k_dot, g, NT, 0, st, (int64_t)n, a, b, d_partials.get(), d_counters.get() + 5, d_norm.get());
  FG_CUDA(cudaMemcpyAsync(h_scalar.get(), d_norm.get(), sizeof(double), cudaMemcpyDeviceToHost, st));
  FG_CUDA(cudaStreamSynchronize(st));
  *out = h_scalar.get()[0];
  return FG_OK;
}

// res = rhs - S z in FP64 arithmetic; returns ||res||.
template <class TS>
fg_status SchurImpl<TS>::reduced_residual_d(double lambda, const double* z, double* res, double* rnorm) {
  if (!retained) { *rnorm = 0; return FG_OK; }
  PView<double> pv{z, nullptr, nullptr};
  FG_TRY(apply_reduced<double>(pv, lambda, lambda, true, d_tmpd.get(), d_qd.get(), nullptr, nullptr));
  unsigned g = std::min<unsigned>(grid_for(retained, NT), 4 * nsm);
  FG_LAUNCH(k_sub_norms, g, NT, 0, st, (int64_t)retained, d_qd.get(), d_rhs.get(), 1.0, res, d_partials.get(),
            d_counters.get() + 6, d_norm.get());
  FG_CUDA(cudaMemcpyAsync(h_scalar.get(), d_norm.get(), 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  FG_CUDA(cudaStreamSynchronize(st));
  *rnorm = std::sqrt(h_scalar.get()[0]);
  return FG_OK;
}

// src/schur.rs:346-397 with src/linear_model.rs:254-282.
template <class TS>
fg_status SchurImpl<TS>::verify(double lambda, double* predicted) {
  Layout L = layout();
  VerifyState* vs = d_ver.get();
  FG_CUDA(cudaMemsetAsync(vs, 0, sizeof(VerifyState), st));
  double red2 = 0, rhs2 = 0;
  const bool known = final_residual_known && retained;
  if (known) {  // the FP32 solve ended on an FP64 residual b - S z of this very z
    red2 = h_pcg.get()->rr_last;
    rhs2 = h_pcg.get()->bnorm * h_pcg.get()->bnorm;
  } else if (retained) {
    PView<double> pv{d_zred.get(), nullptr, nullptr};
    FG_TRY(apply_reduced<double>(pv, lambda, lambda, true, d_tmpd.get(), d_qd.get(), nullptr, nullptr));
    unsigned g = std::min<unsigned>(grid_for(retained, NT), 4 * nsm);
    FG_LAUNCH(k_sub_norms, g, NT, 0, st, (int64_t)retained, d_qd.get(), d_rhs.get(), -1.0, (double*)nullptr,
              d_partials.get(), d_counters.get() + 6, d_norm.get() + 2);
  }
  if (rows) FG_CUDA(cudaMemsetAsync(d_jd.get(), 0, rows * sizeof(double), st));
  if (nemissions && source == DEVICE_BAL && pure_pairs && cw == 9 && pw == 3)
    FG_LAUNCH(k_jdelta_bal<TS>, std::min<unsigned>(grid_for(nemissions, NT), 4 * nsm), NT, 0, st,
              (int64_t)nemissions, (int64_t)retained,
              d_edges.get(), d_values.get(), d_step.get(), d_jd.get(), d_partials.get(), vs);
  else if (nemissions)
    FG_LAUNCH(k_jdelta<TS>, grid_for(nemissions, NT), NT, 0, st, (int64_t)nemissions, d_emi_off.get(), d_blocks.get(),
              d_values.get(), d_step.get(), d_jd.get(), d_partials.get(), vs);
  const bool bal = bal_layout();
  if (nC && bal) {
    FG_LAUNCH((k_bal_cam_pass<TS, BAL_NORMAL>), (unsigned)nC, BAL_CAM_THREADS, 0, st, (int64_t)nC, d_cam_edge_off.get(),
              d_values.get(), d_negres.get(), d_jd.get(), d_camjt.get(), (double*)nullptr);
  } else if (nC) {
    FG_DISPATCH_WIDTHS(cw, pw, {
      FG_LAUNCH((k_cam_jt_block<CW_, TS, CAM_NORMAL>), (unsigned)nC, 128, 0, st, L, d_var_off.get(),
                d_var_blk.get(), d_blocks.get(), d_values.get(), d_negres.get(), d_jd.get(), d_camjt.get());
    });
  }
  if (dim)
    FG_LAUNCH(k_normal_residual<TS>, std::min<unsigned>(grid_for(dim, NT), 4 * nsm), NT, 0, st, L,
              d_var_off.get(), d_var_blk.get(),
              d_blocks.get(), d_values.get(), d_jd.get(), d_negres.get(), d_g.get(), d_scales.get(), d_step.get(),
              lambda, nC ? d_camjt.get() : (const double*)nullptr, d_partials.get() + 4 * 65536, vs,
              bal ? d_pt_edge_off.get() : (const int64_t*)nullptr, bal ? d_pt_edge.get() : (const int64_t*)nullptr);
  FG_CUDA(cudaMemcpyAsync(h_ver.get(), vs, sizeof(VerifyState), cudaMemcpyDeviceToHost, st));
  if (coarse_on)  // whether the coarse matrix of this solve was positive definite
    FG_CUDA(cudaMemcpyAsync(h_count.get() + 3, d_coarse_ok.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
  if (retained && !known)
    FG_CUDA(cudaMemcpyAsync(h_scalar.get() + 2, d_norm.get() + 2, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  FG_CUDA(cudaStreamSynchronize(st));
  if (retained && !known) { red2 = h_scalar.get()[2]; rhs2 = h_scalar.get()[3]; }
  if (coarse_on && h_count.get()[3] == 0) diag.coarse_vectors = 0;
  const VerifyState& v = *h_ver.get();
  auto rel = [](double n, double r) { return r == 0 ? n : n / r; };
  diag.reduced_relative_residual = rel(std::sqrt(red2), std::sqrt(rhs2));
  diag.has_reduced = 1;
  diag.original_relative_residual = rel(std::sqrt(v.nr2), std::sqrt(v.g2));
  diag.has_original = 1;
  diag.scaled_relative_residual = rel(std::sqrt(v.snr2), std::sqrt(v.sg2));
  diag.has_scaled = 1;
  double pred = -v.gd - 0.5 * v.jd2;
  bool bad = v.nonfinite_step || !std::isfinite(pred) || !std::isfinite(diag.reduced_relative_residual) ||
             !std::isfinite(diag.original_relative_residual) || !std::isfinite(diag.scaled_relative_residual) ||
             (diag.has_estimated && !std::isfinite(diag.estimated_relative_residual));
  if (bad) {
    diag.termination = FG_TERM_NONFINITE;
    set_error("nonfinite step or residual");
    return FG_LINEAR_SOLVE_FAILED;
  }
  *predicted = pred;
  return FG_OK;
}

}  // namespace fg
