// Kernel-shape autotuner (TS_PLAN_AUTOTUNE).
//
// The shapes that decide a plan's speed depend on the grid and the GPU: the
// tensor-core tiles (latitudes per synthesis tile, degrees per analysis
// tile: operand reuse against pipeline depth and tile count), the FFT's
// radix split H = P*Q (the in-register DFT lengths of its two phases) and
// its rows per CTA (occupancy against shared memory).  With TS_PLAN_AUTOTUNE the
// plan times every candidate on a scratch batch at creation, keeps the
// fastest, and remembers the choice for later plans of the same grid on the
// same kind of device in this process.  The scratch batch holds zeros: the
// kernels' work does not depend on the values.
#include <map>
#include <mutex>
#include <string>

#include "runtime.h"

namespace {

struct Shapes {
  int nl = 0, ltl = 0, rows = 0;
  bool alt = false;  // the FFT's second P*Q split
};

std::mutex g_mu;
std::map<std::string, Shapes> g_cache;

std::string cache_key(ts_plan p) {
  char buf[256];
  snprintf(buf, sizeof buf, "%s|%d|%d|%d|%d|%d|%d", p->ctx->name.c_str(), p->lmax, p->mmax,
           p->nlat, p->nphi, p->precision, p->fourier);
  return buf;
}

// device scratch of the timing batch
struct Scratch {
  float *q = nullptr, *spat = nullptr, *fm = nullptr;
  char *img = nullptr;
  ~Scratch() {
    for (void *x : {(void *)q, (void *)spat, (void *)fm, (void *)img})
      if (x) cudaFree(x);
  }
};

// mean device time of `reps` runs after two untimed ones
template <class F>
float time_ms(cudaStream_t s, F &&run, int reps = 4) {
  cudaEvent_t a, b;
  TS_CUDA(cudaEventCreate(&a));
  TS_CUDA(cudaEventCreate(&b));
  run();
  run();
  TS_CUDA(cudaEventRecord(a, s));
  for (int i = 0; i < reps; i++) run();
  TS_CUDA(cudaEventRecord(b, s));
  TS_CUDA(cudaEventSynchronize(b));
  float ms = 0;
  TS_CUDA(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms / reps;
}

}  // namespace

void ts_autotune(ts_plan p) {
  const std::string key = cache_key(p);
  {
    std::lock_guard<std::mutex> lock(g_mu);
    auto it = g_cache.find(key);
    if (it != g_cache.end()) {
      const bool tc_changes = p->tc && (it->second.nl != p->tune_nl || it->second.ltl != p->tune_ltl);
      p->tune_nl = it->second.nl;
      p->tune_ltl = it->second.ltl;
      p->fft_rows = it->second.rows;
      p->fft_alt = it->second.alt;
      if (tc_changes) {
        ts_tc_free(p);
        ts_tc_init(p);
      }
      p->tuned = true;
      return;
    }
  }
  cudaStream_t s = p->ctx->stream;
  // timing batch: up to 128 fields, at most ~512 MB of grid
  const size_t grid_bytes = sizeof(float) * (size_t)p->nlat * p->nphi;
  const int B = (int)std::max<size_t>(8, std::min<size_t>(128, (512u << 20) / grid_bytes));
  const long fm_stride = (long)(p->mmax + 1) * p->nlat;
  Scratch sc;
  TS_CUDA(cudaMalloc(&sc.q, sizeof(float2) * p->nlm * B));
  TS_CUDA(cudaMalloc(&sc.spat, grid_bytes * B));
  TS_CUDA(cudaMalloc(&sc.fm, sizeof(float2) * fm_stride * B));
  TS_CUDA(cudaMemsetAsync(sc.q, 0, sizeof(float2) * p->nlm * B, s));
  TS_CUDA(cudaMemsetAsync(sc.spat, 0, grid_bytes * B, s));
  TS_CUDA(cudaMemsetAsync(sc.fm, 0, sizeof(float2) * fm_stride * B, s));

  Shapes best;
  // tensor-core tiles
  if (p->precision != TS_PREC_FP32) {
    const size_t img_bytes = ts_tc_wimg_bytes(p, B, TS_TC_FIELDS);
    TS_CUDA(cudaMalloc(&sc.img, img_bytes));
    TS_CUDA(cudaMemsetAsync(sc.img, 0, img_bytes, s));
    TsFields qf{};
    qf.base[0] = (const float2 *)sc.q;
    qf.inst_stride[0] = p->nlm;
    qf.nper = 1;
    float best_ms = 1e30f;
    std::vector<std::pair<int, int>> seen;
    for (int nl : {64, 96})
      for (int ltl : {64, 128}) {
        p->tune_nl = nl;
        p->tune_ltl = ltl;
        const TsTcGeom g = ts_tc_geom(p);  // candidates collapse on small grids
        bool dup = false;
        for (auto &pr : seen) dup = dup || (pr.first == g.NL && pr.second == g.LTL);
        if (dup) continue;
        seen.push_back({g.NL, g.LTL});
        ts_tc_free(p);
        ts_tc_init(p);
        const float ms = time_ms(s, [&] {
          ts_launch_leg_synth_tc(p, qf, (float2 *)sc.fm, fm_stride, B, s);
          ts_launch_analys_tc_img(p, sc.img, B, (float2 *)sc.q, p->nlm, s);
        });
        if (ms < best_ms) {
          best_ms = ms;
          best.nl = g.NL;
          best.ltl = g.LTL;
        }
      }
    p->tune_nl = best.nl;
    p->tune_ltl = best.ltl;
    if (!seen.empty() && (seen.back().first != best.nl || seen.back().second != best.ltl)) {
      ts_tc_free(p);
      ts_tc_init(p);
    }
  }
  // FFT: the P*Q split (the default, and the second one where the row
  // length has one) and the rows per CTA of each
  int P, Q;
  if (ts_f2_shape(p, &P, &Q)) {
    float best_ms = 1e30f;
    const bool has_alt = ts_f2_has_alt(p);
    for (int alt = 0; alt <= (has_alt ? 1 : 0); alt++) {
     p->fft_alt = alt != 0;
     int rows_seen[2] = {0, 0}, n = 0;
     for (int rows : {8, 16, 4}) {
      p->fft_rows = rows;
      const int r = ts_f2_rows(p);
      if (r == rows_seen[0] || r == rows_seen[1] || n == 2) continue;
      rows_seen[n++] = r;
      const float ms = time_ms(s, [&] {
        ts_launch_fourier_synth(p, (const float2 *)sc.fm, fm_stride, sc.spat,
                                (long)p->nlat * p->nphi, B, s);
        if (p->precision != TS_PREC_FP32)
          ts_launch_fourier_analys_w(p, sc.spat, (long)p->nlat * p->nphi, B, TS_TC_FIELDS,
                                     sc.img, s);
        else
          ts_launch_fourier_analys(p, sc.spat, (long)p->nlat * p->nphi, (float2 *)sc.fm,
                                   fm_stride, B, s);
      });
      if (ms < best_ms) {
        best_ms = ms;
        best.rows = r;
        best.alt = alt != 0;
      }
     }
    }
    p->fft_rows = best.rows;
    p->fft_alt = best.alt;
  }
  TS_CUDA(cudaStreamSynchronize(s));
  p->tuned = true;
  std::lock_guard<std::mutex> lock(g_mu);
  g_cache[key] = best;
}
