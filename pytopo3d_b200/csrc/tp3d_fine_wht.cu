// Launch side of the Walsh-Hadamard fine operator (tp3d_fine_wht.cuh):
// explicit instantiations per precision, modulus source, epilogue mode and
// block shape; the KE block split; the tile chooser.
#include <algorithm>
#include <cmath>
#include <vector>

#include "tp3d_fine_wht.cuh"
#include "tp3d_fine_wht1.cuh"
#include "tp3d_fine_wht2.cuh"

namespace tp3d {

namespace {

// (threads, min blocks per SM, kernel) of each variant, per precision.
// Kernels: 0 the scalar two-barrier kernel (tp3d_fine_wht.cuh), 1 the packed
// FP32 two-plane kernel (tp3d_fine_wht2.cuh, twice the scalar kernel's
// per-thread state, so fewer threads per block), 2 the one-barrier kernel
// (tp3d_fine_wht1.cuh) for the epilogue modes of wht1_mode() and the
// two-barrier kernel for the others (same tile, same results).  The timed
// choice considers kernels 0 and 2.
enum : int { kWhtScalar = 0, kWhtPacked = 1, kWhtOneBarrier = 2 };
template <typename T>
struct WhtShapes;
template <>
struct WhtShapes<float> {
  static constexpr int count = 8;
  static constexpr int nthr[kWhtVariants] = {256, 384, 128, 512, 768, 256, 256, 512};
  static constexpr int minb[kWhtVariants] = {1, 1, 3, 2, 1, 4, 4, 2};
  static constexpr int kind[kWhtVariants] = {kWhtPacked, kWhtPacked, kWhtPacked,     kWhtScalar,
                                             kWhtScalar, kWhtScalar, kWhtOneBarrier, kWhtOneBarrier};
};
template <>
struct WhtShapes<double> {
  static constexpr int count = 3;
  static constexpr int nthr[kWhtVariants] = {256, 384, 128, 256, 256, 256, 256, 256};
  static constexpr int minb[kWhtVariants] = {2, 1, 4, 2, 2, 2, 2, 2};
  static constexpr int kind[kWhtVariants] = {kWhtScalar, kWhtScalar, kWhtScalar, kWhtScalar,
                                             kWhtScalar, kWhtScalar, kWhtScalar, kWhtScalar};
};

// Epilogue modes that the one-barrier shapes run in the one-barrier kernel:
// the plain apply, the residual, the CG product and the power-iteration step.
// The Chebyshev and Jacobi steps (up to nine epilogue inputs per node) spill
// in it under 64 registers per thread and measured faster in the two-barrier
// kernel (128x64x64 SIMP step: 8.98 ms with this split, 9.10 ms with every
// mode in the one-barrier kernel, 9.02 ms with none).
constexpr bool wht1_mode(int mode) {
  return mode == kModeApply || mode == kModeResid || mode == kModeCgQ || mode == kModeDinvApply;
}

// dynamic shared memory of a launch of variant v
template <typename T>
constexpr size_t wht_kernel_smem(int v) {
  const int k = WhtShapes<T>::kind[v], n = WhtShapes<T>::nthr[v];
  return k == kWhtPacked ? wht2_smem_bytes(n) : (k == kWhtOneBarrier ? wht1_smem_bytes<T>(n) : wht_smem_bytes<T>(n));
}

template <typename T, class ESrc, int V>
struct WhtVariant {
  static constexpr int NTHR = WhtShapes<T>::nthr[V];
  static constexpr int MINB = WhtShapes<T>::minb[V];
  template <int MODE>
  static void* fn() {
    constexpr int K = WhtShapes<T>::kind[V];
    if constexpr (K == kWhtPacked) return (void*)wht2_apply_kernel<ESrc, MODE, NTHR, MINB>;
    else if constexpr (K == kWhtOneBarrier && wht1_mode(MODE))
      return (void*)wht1_apply_kernel<T, ESrc, MODE, NTHR, MINB>;
    else return (void*)wht_apply_kernel<T, ESrc, MODE, NTHR, MINB>;
  }
  static void* by_mode(int mode) {
    switch (mode) {
      case kModeApply: return fn<kModeApply>();
      case kModeResid: return fn<kModeResid>();
      case kModeJacobi: return fn<kModeJacobi>();
      case kModeCgQ: return fn<kModeCgQ>();
      case kModeChebFirst: return fn<kModeChebFirst>();
      case kModeChebStep: return fn<kModeChebStep>();
      case kModeChebStepDot: return fn<kModeChebStepDot>();
      default: return fn<kModeDinvApply>();
    }
  }
};

template <typename T, class ESrc>
void* wht_fn(int mode, int v) {
  if constexpr (WhtShapes<T>::count > 3) {
    switch (v) {
      case 3: return WhtVariant<T, ESrc, 3>::by_mode(mode);
      case 4: return WhtVariant<T, ESrc, 4>::by_mode(mode);
      case 5: return WhtVariant<T, ESrc, 5>::by_mode(mode);
      case 6: return WhtVariant<T, ESrc, 6>::by_mode(mode);
      case 7: return WhtVariant<T, ESrc, 7>::by_mode(mode);
      default: break;
    }
  }
  switch (v) {
    case 0: return WhtVariant<T, ESrc, 0>::by_mode(mode);
    case 1: return WhtVariant<T, ESrc, 1>::by_mode(mode);
    default: return WhtVariant<T, ESrc, 2>::by_mode(mode);
  }
}

// dynamic shared memory of every instantiation raised once to what it needs
template <typename T, class ESrc>
bool wht_prepare(int v) {
  const int nthr = WhtShapes<T>::nthr[v];
  const int smem = (int)wht_kernel_smem<T>(v);
  for (int mode = 0; mode <= kModeChebStepDot; ++mode)
    if (ensure_dynamic_smem(wht_fn<T, ESrc>(mode, v), smem) != TP3D_OK) return false;
  return true;
}

}  // namespace

template <typename T, class ESrc>
int wht_variant_threads(int v) {
  return WhtShapes<T>::nthr[v];
}

template <typename T, class ESrc>
int wht_variant_count() {
  return WhtShapes<T>::count;
}

template <typename T, class ESrc>
bool wht_variant_timed(int v) {
  return v >= 0 && v < WhtShapes<T>::count && WhtShapes<T>::kind[v] != kWhtPacked;
}

template <typename T, class ESrc>
int wht_occupancy(int v) {
  if (!wht_prepare<T, ESrc>(v)) return 1;
  int occ = 0;
  const int nthr = WhtShapes<T>::nthr[v];
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, wht_fn<T, ESrc>(kModeChebStep, v), nthr,
                                                wht_kernel_smem<T>(v));
  return std::max(occ, 1);
}

template <typename T, class ESrc>
int wht_launch(const WhtParams<T, ESrc>& p, int mode, int v, dim3 grid, cudaStream_t st, bool pdl) {
  if (v < 0 || v >= WhtShapes<T>::count || !wht_prepare<T, ESrc>(v)) return TP3D_ERR_ARG;
  const int nthr = WhtShapes<T>::nthr[v];
  void* args[] = {(void*)&p};
  const cudaError_t e = launch_kernel_c(pdl, wht_fn<T, ESrc>(mode, v), grid, dim3(nthr), wht_kernel_smem<T>(v),
                                        st, args);
  return e == cudaSuccess ? TP3D_OK : TP3D_ERR_CUDA;
}

bool wht_blocks_from_ke(const double* KE, double m[8][3][3]) {
  // W[(s, i), (a, i)] = (-1)^(s . offset(a)), s = sx + 2 sy + 4 sz
  auto sgn = [](int s, int a) {
    const int d = (s & 1) * corner_ox(a) + ((s >> 1) & 1) * corner_oy(a) + ((s >> 2) & 1) * corner_oz(a);
    return (d & 1) ? -1.0 : 1.0;
  };
  double mx = 0.0;
  for (int i = 0; i < 576; ++i) mx = std::max(mx, std::fabs(KE[i]));
  if (!(mx > 0.0)) return false;
  // Mfull = W KE W^T / 64
  static double Mf[24][24];
  for (int s1 = 0; s1 < 8; ++s1)
    for (int i = 0; i < 3; ++i)
      for (int s2 = 0; s2 < 8; ++s2)
        for (int j = 0; j < 3; ++j) {
          double acc = 0.0;
          for (int a = 0; a < 8; ++a)
            for (int b = 0; b < 8; ++b) acc += sgn(s1, a) * sgn(s2, b) * KE[(3 * a + i) * 24 + 3 * b + j];
          Mf[3 * s1 + i][3 * s2 + j] = acc / 64.0;
        }
  const double tol = 1e-12 * mx;
  for (int s1 = 0; s1 < 8; ++s1)
    for (int i = 0; i < 3; ++i)
      for (int s2 = 0; s2 < 8; ++s2)
        for (int j = 0; j < 3; ++j) {
          const bool in_block = (s1 ^ (1 << i)) == (s2 ^ (1 << j));
          const bool translation = s1 == 0 || s2 == 0;
          if ((!in_block || translation) && std::fabs(Mf[3 * s1 + i][3 * s2 + j]) > tol) return false;
        }
  for (int t = 0; t < 8; ++t)
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) m[t][i][j] = Mf[3 * (t ^ (1 << i)) + i][3 * (t ^ (1 << j)) + j];
  return true;
}

// The patch is PY = TY + 2 threads along y (the contiguous direction) by
// TX + 2 along x.  Tile candidates are ranked by blocks per node plane (the
// fewest first: the fewest halo threads), ties by the larger tile; each gets
// the number of z chunks that minimises the busiest SM's work, counting each
// block's prologue as 1.5 planes and crediting co-resident blocks for hiding
// each other's barrier and memory latency.
template <typename T, class ESrc>
int wht_tile_candidates(const Grid& g, int nsm, int v, WhtTile* out, int max_out) {
  const int NX = g.nx + 1, NY = g.ny + 1, NZ = g.nz + 1;
  const int nthr = WhtShapes<T>::nthr[v];
  const int occ = wht_occupancy<T, ESrc>(v);
  struct Cand {
    long long blocks;
    int area, PY;
  };
  std::vector<Cand> cands;
  for (int PY = 4; PY <= std::min(nthr / 4, NY + 2); ++PY) {
    const int TY = PY - 2, TX = nthr / PY - 2;
    if (TX < 2) continue;
    const long long blocks = (long long)((NY + TY - 1) / TY) * ((NX + TX - 1) / TX);
    cands.push_back({blocks, TX * TY, PY});
  }
  std::sort(cands.begin(), cands.end(), [](const Cand& x, const Cand& y) {
    return x.blocks != y.blocks ? x.blocks < y.blocks : (x.area != y.area ? x.area > y.area : x.PY < y.PY);
  });
  auto eff = [&](long long L) {
    const long long l = std::min<long long>(L, occ);
    return l <= 1 ? 1.0 : (l == 2 ? 1.6 : (l == 3 ? 1.85 : 2.0));
  };
  int n = 0;
  for (const Cand& c : cands) {
    if (n >= max_out) break;
    WhtTile t;
    t.variant = v;
    t.nthr = nthr;
    t.occ = occ;
    t.PY = c.PY;
    t.TY = c.PY - 2;
    t.TX = nthr / c.PY - 2;
    t.tiles_y = (NY + t.TY - 1) / t.TY;
    t.tiles_x = (NX + t.TX - 1) / t.TX;
    double best_t = 1e300;
    for (int zc = 1; zc <= NZ; ++zc) {
      const long long nch = (NZ + zc - 1) / zc;
      if ((nch - 1) * zc >= NZ) continue;
      const long long per_sm = (c.blocks * nch + nsm - 1) / nsm;
      const double tm = (double)per_sm * (zc + 1.5) / eff(per_sm);
      if (tm < best_t - 1e-9) {
        best_t = tm;
        t.ZC = zc;
        t.zchunks = (int)nch;
      }
    }
    out[n++] = t;
  }
  return n;
}

template <typename T, class ESrc>
WhtTile wht_choose_tile(const Grid& g, int nsm, int v) {
  WhtTile t;
  t.variant = v;
  t.nthr = WhtShapes<T>::nthr[v];
  wht_tile_candidates<T, ESrc>(g, nsm, v, &t, 1);
  return t;
}

#define TP3D_WHT_INSTANTIATE(T, ESrc)                                                     \
  template int wht_variant_threads<T, ESrc>(int);                                        \
  template int wht_variant_count<T, ESrc>();                                             \
  template bool wht_variant_timed<T, ESrc>(int);                                         \
  template int wht_occupancy<T, ESrc>(int);                                              \
  template int wht_launch<T, ESrc>(const WhtParams<T, ESrc>&, int, int, dim3, cudaStream_t, bool); \
  template WhtTile wht_choose_tile<T, ESrc>(const Grid&, int, int);                     \
  template int wht_tile_candidates<T, ESrc>(const Grid&, int, int, WhtTile*, int);
TP3D_WHT_INSTANTIATE(double, EFromF64)
TP3D_WHT_INSTANTIATE(float, EFromF32)
TP3D_WHT_INSTANTIATE(float, EFromBF16)
#undef TP3D_WHT_INSTANTIATE

}  // namespace tp3d
