// C ABI (include/exahype_b200.h): template dispatch over (dimension, order,
// PDE), operator-table upload, and the uniform-mesh solver that sequences the
// kernels like the reference's non-fused time step.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cfloat>
#include <climits>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/exahype_b200.h"
#include "aderdg.cuh"
#include "predictor_lines.cuh"
#include "limiter.cuh"
#include "linear.cuh"
#include "amr.cuh"

namespace exa {

static thread_local std::string g_last_error;

static int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define EXA_CUDA(call)                                                                               \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess) return fail(EXA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define EXA_LAUNCHED()                                                                                     \
  do {                                                                                                     \
    cudaError_t e_ = cudaGetLastError();                                                                   \
    if (e_ != cudaSuccess) return fail(EXA_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e_)); \
  } while (0)

// Stream-ordered device allocation for the meshes: cudaMallocAsync and
// cudaFreeAsync on the owner's stream never wait for other streams (cudaFree
// synchronises the whole device), so creating or destroying one mesh does
// not stall the work queued for others.
// The memory comes from a pool of the library's own per device that keeps
// freed memory for reuse instead of returning it to the driver, so a server
// that creates and destroys meshes continuously does not pay for it each time.
static cudaMemPool_t library_pool() {
  static std::mutex mu;
  static std::vector<std::pair<int, cudaMemPool_t>> pools;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  for (const auto& e : pools)
    if (e.first == dev) return e.second;
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = dev;
  cudaMemPool_t pool = nullptr;
  if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
  uint64_t keep = UINT64_MAX;
  cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  pools.emplace_back(dev, pool);
  return pool;
}
template <class T>
static bool salloc(T** p, size_t bytes, cudaStream_t st) {
  cudaMemPool_t pool = library_pool();
  if (!pool) return false;
  return cudaMallocFromPoolAsync(reinterpret_cast<void**>(p), bytes, pool, st) == cudaSuccess;
}
static void sfree(void* p, cudaStream_t st) {
  if (p) cudaFreeAsync(p, st);
}

// ---- tables ---------------------------------------------------------------
static int upload_tables() {
  static std::mutex mu;
  static std::vector<int> done_dev;
  int dev = 0;
  EXA_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  for (int d : done_dev)
    if (d == dev) return EXA_OK;
  std::vector<OrderTables> h(kMaxOrder + 1);
  std::vector<LimiterTables> hl(kMaxOrder + 1);
  std::vector<double> afine(3 * kAmrSq, 0.0), arestr(3 * kAmrSq, 0.0), aequi(kAmrSq, 0.0);
  std::memset(h.data(), 0, sizeof(OrderTables) * h.size());
  std::memset(hl.data(), 0, sizeof(LimiterTables) * hl.size());

  for (int N = 1; N <= kMaxOrder; N++) {
    const int b = N + 1, bl = 2 * N + 1;
    OrderTables& t = h[N];
    LimiterTables& l = hl[N];
    for (int i = 0; i < b; i++) {
      t.w[i] = exa_tab_weights[exa_tab_weights_off[N] + i];
      t.x[i] = exa_tab_nodes[exa_tab_nodes_off[N] + i];
      t.FL[i] = exa_tab_FLCoeff[exa_tab_FLCoeff_off[N] + i];
      t.FR[i] = exa_tab_FRCoeff[exa_tab_FRCoeff_off[N] + i];
      t.lobatto[i] = exa_tab_lobatto_nodes[exa_tab_lobatto_nodes_off[N] + i];
    }
    for (int i = 0; i < b * b; i++) {
      t.Kxi[i] = exa_tab_Kxi[exa_tab_Kxi_off[N] + i];
      t.iK1[i] = exa_tab_iK1[exa_tab_iK1_off[N] + i];
      t.dudx[i] = exa_tab_dudx[exa_tab_dudx_off[N] + i];
      t.Kxi_f[i] = (float)t.Kxi[i];
      l.uh2lob[i] = exa_tab_uh2lob[exa_tab_uh2lob_off[N] + i];
    }
    if (b % 2 == 0) {
      const int hh = b / 2;
      for (int n = 0; n < hh; n++)
        for (int m = 0; m < hh; m++) {
          t.KxiP[n * hh + m] = 0.5 * (t.Kxi[n * b + m] + t.Kxi[(b - 1 - n) * b + m]);
          t.KxiQ[n * hh + m] = 0.5 * (t.Kxi[n * b + m] - t.Kxi[(b - 1 - n) * b + m]);
        }
    }
    for (int i = 0; i < b * bl; i++) {
      l.uh2lim[i] = exa_tab_uh2lim[exa_tab_uh2lim_off[N] + i];
      l.lim2uh[i] = exa_tab_lim2uh[exa_tab_lim2uh_off[N] + i];
    }
    double* fine = afine.data() + 3 * amr_off(N);
    for (int i = 0; i < 3 * b * b; i++) fine[i] = exa_tab_fineGridProjector1d[exa_tab_fineGridProjector1d_off[N] + i];
    for (int j = 0; j < 3; j++)
      for (int m = 0; m < b; m++)
        for (int n = 0; n < b; n++)
          arestr[3 * amr_off(N) + (j * b + m) * b + n] = t.w[n] * fine[(j * b + m) * b + n] / (3.0 * t.w[m]);
    for (int i = 0; i < b * b; i++)
      aequi[amr_off(N) + i] = exa_tab_equidistantGridProjector1d[exa_tab_equidistantGridProjector1d_off[N] + i];
  }
  EXA_CUDA(cudaMemcpyToSymbol(c_tab, h.data(), sizeof(OrderTables) * h.size()));
  EXA_CUDA(cudaMemcpyToSymbol(g_lim_tab, hl.data(), sizeof(LimiterTables) * hl.size()));
  EXA_CUDA(cudaMemcpyToSymbol(c_amr_fine, afine.data(), sizeof(double) * afine.size()));
  EXA_CUDA(cudaMemcpyToSymbol(c_amr_restr, arestr.data(), sizeof(double) * arestr.size()));
  EXA_CUDA(cudaMemcpyToSymbol(c_amr_equi, aequi.data(), sizeof(double) * aequi.size()));
  done_dev.push_back(dev);
  return EXA_OK;
}

// ---- per-(DIM, N, PDE) launchers ------------------------------------------
struct KernelSet {
  int dim, order, pde, nvar, npar, P, F;
  bool linear;  // linear PDE: Cauchy-Kovalevski predictor, linear Riemann solver and surface integral
  // (luh, lQhbnd, lFhbnd, lduh, iters, dt, geo, n, list, count, temps, with_temps, sweeps, variant, stream);
  // count (optional, device) caps the list length at launch time
  int (*predictor)(const double*, double*, double*, double*, int*, const double*, Geometry, int, const int*,
                   const int*, PredictorTemps, bool, unsigned long long*, int, cudaStream_t);
  // the last pointer before the stream: optional device gate (0 skips the work)
  int (*riemann)(const double*, double*, const int*, const int*, const int*, int, const int*, cudaStream_t);
  int (*boundary)(const double*, double*, const int*, const int*, int, int, const int*, cudaStream_t);
  int (*corrector)(double*, const double*, const double*, const double*, double*, Geometry, int, const int*, int,
                   const int*, cudaStream_t);
  // volumeIntegralLinear on its own (lduh, lFhi, ncells, stream); linear PDEs only
  int (*volume)(double*, const double*, int, cudaStream_t);
  // AMR transfers (op 0 prolongation, 1 restriction): volume (a, b, n, fine,
  // coarse, levelDelta, index[3n], op, stream) and face (state a, flux a,
  // state b, flux b, n, fine slot, coarse slot, levelDelta, index[2n], op,
  // stream); plot vertices (luh, out, ncells, stream)
  int (*amr_volume)(double*, const double*, int, const int*, const int*, const int*, const int*, int, cudaStream_t);
  int (*amr_face)(double*, double*, const double*, const double*, int, const int*, const int*, const int*,
                  const int*, int, cudaStream_t);
  int (*plot)(const double*, double*, int, cudaStream_t);
  bool point_source;  // the PDE has a point source (usePointSource)
};

template <int DIM, int N, class PDE>
struct AmrLaunch {
  static constexpr int ND = PDE::nVar + PDE::nPar, NV = PDE::nVar;
  static int volume(double* a, const double* b, int n, const int* fine, const int* coarse, const int* ld,
                    const int* idx, int op, cudaStream_t st) {
    if (n <= 0) return EXA_OK;
    amr_volume_kernel<DIM, N, ND><<<n, 128, 0, st>>>(a, b, n, fine, coarse, ld, idx, op);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static int face(double* qa, double* fa, const double* qb, const double* fb, int n, const int* fine,
                  const int* coarse, const int* ld, const int* idx, int op, cudaStream_t st) {
    if (n <= 0) return EXA_OK;
    amr_face_kernel<DIM, N, ND, NV><<<n, 256, 0, st>>>(qa, fa, qb, fb, n, fine, coarse, ld, idx, op);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static int plot(const double* luh, double* out, int n, cudaStream_t st) {
    if (n <= 0) return EXA_OK;
    plot_vertex_kernel<DIM, N, ND><<<n, 256, 0, st>>>(luh, out, n);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static void fill(KernelSet& k) {
    k.amr_volume = &volume;
    k.amr_face = &face;
    k.plot = &plot;
  }
};

template <int DIM, int N, class PDE>
__global__ void sweep_count_kernel(const int* iters, const int* cell_list, int n, const int* count,
                                   unsigned long long* acc) {
  if (count) n = min(n, *count);
  unsigned long long s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += (unsigned long long)iters[cell_list ? cell_list[i] : i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(acc, s);
}

template <int DIM, int N, class PDE>
static int launch_corrector(double* luh, const double* du, const double* fb, const double* dt, double* dtout,
                            Geometry g, int n, const int* list, int upd, const int* cnt, cudaStream_t st) {
  using CC = CorrectorCfg<DIM, N, PDE>;
  if (n <= 0) return EXA_OK;
  static bool attr = false;
  if (!attr) {
    EXA_CUDA(cudaFuncSetAttribute(corrector_kernel<DIM, N, PDE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)CC::SMEM));
    attr = true;
  }
  corrector_kernel<DIM, N, PDE><<<(n + CC::CPB - 1) / CC::CPB, CC::THREADS, CC::SMEM, st>>>(luh, du, fb, dt, dtout, g,
                                                                                           n, list, upd, cnt);
  EXA_LAUNCHED();
  return EXA_OK;
}

// Predictor variants the autotuner chooses from (all FP64):
//   0 node form, 1 block/SM budget    1 line form, 1 block/SM
//   2 line form, 2 blocks/SM          3 node form, 2 blocks/SM
//   6 line form, two time slices per phase, 2 blocks/SM
//   7 line form, two time slices per phase, 1 block/SM
//   8 line form, Picard iterate in tensor memory, two slices per phase,
//     2 blocks/SM (orders up to 5 with five state variables; elsewhere as
//     variant 6)
// and the mixed-precision line form (FP32 increment sweeps after the first
// FP64 sweep), selected explicitly, never by the autotuner:
//   4 mixed line form, 1 block/SM     5 mixed line form, 2 blocks/SM
constexpr int kAllVariants = 9;
constexpr bool variant_is_mixed(int v) { return v == 4 || v == 5; }

template <int DIM, int N, class PDE>
struct Launch {
  using CC = CorrectorCfg<DIM, N, PDE>;

  template <bool TEMPS, int VS, int MB>
  static int launch_pred(const double* luh, double* qb, double* fb, double* du, int* iters, const double* dt,
                         Geometry g, int n, const int* list, const int* cnt, PredictorTemps tmp, cudaStream_t st) {
    using PC = PredictorCfg<DIM, N, PDE, VS, MB>;
    static bool attr = false;
    if (!attr) {
      EXA_CUDA(cudaFuncSetAttribute(predictor_kernel<DIM, N, PDE, TEMPS, VS, MB>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PC::SMEM));
      attr = true;
    }
    const int grid = (n + PC::CPB - 1) / PC::CPB;
    predictor_kernel<DIM, N, PDE, TEMPS, VS, MB><<<grid, PC::THREADS, PC::SMEM, st>>>(luh, qb, fb, du, iters, dt, g,
                                                                                     n, list, tmp, cnt);
    EXA_LAUNCHED();
    return EXA_OK;
  }

  template <bool TEMPS, int MB, bool MIXED = false, int TS = 1, bool TM = false>
  static int launch_lines(const double* luh, double* qb, double* fb, double* du, int* iters, const double* dt,
                          Geometry g, int n, const int* list, const int* cnt, PredictorTemps tmp, cudaStream_t st) {
    using LC = LinesCfg<DIM, N, PDE, MB, MIXED, TS, TM>;
    static bool attr = false;
    if (!attr) {
      EXA_CUDA(cudaFuncSetAttribute(predictor_lines_kernel<DIM, N, PDE, TEMPS, MB, MIXED, TS, TM>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LC::SMEM));
      attr = true;
    }
    const int grid = (n + LC::CPB - 1) / LC::CPB;
    predictor_lines_kernel<DIM, N, PDE, TEMPS, MB, MIXED, TS, TM>
        <<<grid, LC::THREADS, LC::SMEM, st>>>(luh, qb, fb, du, iters, dt, g, n, list, tmp, cnt);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  // two blocks of the line form only fit when their shared memory does
  static constexpr bool kLines2 = 2 * LinesCfg<DIM, N, PDE, 2>::SMEM <= 227 * 1024;
  static constexpr bool kMixed2 = 2 * LinesCfg<DIM, N, PDE, 2, true>::SMEM <= 227 * 1024;
  static constexpr bool kSlices2 = 2 * LinesCfg<DIM, N, PDE, 2, false, 2>::SMEM <= 227 * 1024;
  static constexpr bool kSlices1 = LinesCfg<DIM, N, PDE, 1, false, 2>::SMEM <= 227 * 1024;
  // the tensor-memory iterate (variant 8): five doubles per node and slice
  // (at most 60 columns: N <= 5), a block of whole warps of at most 256 threads
  using Sh = Shape<DIM, N, PDE>;
  static constexpr bool kTmemShape = Sh::nD == 5 && Sh::nV == 5 &&
                                     (cells_per_block<Sh::P>() * Sh::P + 31) / 32 * 32 <= 256 &&
                                     2 * Sh::b * Sh::nD <= 64;
  template <int TS>
  static constexpr bool tmem_fits() {
    if constexpr (kTmemShape) return 2 * LinesCfg<DIM, N, PDE, 2, false, TS, true>::SMEM <= 227 * 1024;
    else return false;
  }
  static constexpr bool kTmem2 = tmem_fits<2>();

  static int predictor(const double* luh, double* qb, double* fb, double* du, int* iters, const double* dt,
                       Geometry g, int n, const int* list, const int* cnt, PredictorTemps tmp, bool temps,
                       unsigned long long* acc, int variant, cudaStream_t st) {
    if (n <= 0) return EXA_OK;
    int rc;
    if constexpr (PDE::kSource || PDE::kNCP)  // source terms: the node form (1 or 2 blocks per SM)
      rc = temps ? launch_pred<true, 1, 1>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st)
           : variant == 3 ? launch_pred<false, 1, 2>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st)
                          : launch_pred<false, 1, 1>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st);
    else if (temps)
      rc = variant == 1 || variant == 2 ? launch_lines<true, 1>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st)
                                        : launch_pred<true, 1, 1>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st);
    else if (variant == 1 || (variant == 2 && !kLines2))
      rc = launch_lines<false, 1>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st);
    else if (variant == 2)
      rc = launch_lines<false, kLines2 ? 2 : 1>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st);
    else if (variant == 3)
      rc = launch_pred<false, 1, 2>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st);
    else if (variant == 4 || (variant == 5 && !kMixed2))
      rc = launch_lines<false, 1, true>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st);
    else if (variant == 5)
      rc = launch_lines<false, kMixed2 ? 2 : 1, true>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st);
    else if (variant == 8 && kTmem2)
      rc = launch_lines<false, 2, false, 2, kTmem2>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st);
    else if ((variant == 6 || variant == 8) && kSlices2)
      rc = launch_lines<false, 2, false, kSlices2 ? 2 : 1>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st);
    else if (variant == 6 || variant == 7 || variant == 8)
      rc = launch_lines<false, 1, false, kSlices1 ? 2 : 1>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st);
    else
      rc = launch_pred<false, 1, 1>(luh, qb, fb, du, iters, dt, g, n, list, cnt, tmp, st);
    if (rc) return rc;
    if (acc && iters) {
      sweep_count_kernel<DIM, N, PDE><<<std::min(1024, (n + 255) / 256), 256, 0, st>>>(iters, list, n, cnt, acc);
      EXA_LAUNCHED();
    }
    return EXA_OK;
  }
  static int riemann(const double* qb, double* fb, const int* l, const int* r, const int* d, int n, const int* gate,
                     cudaStream_t st) {
    if (n <= 0) return EXA_OK;
    riemann_kernel<DIM, N, PDE><<<(n + 3) / 4, 128, 0, st>>>(qb, fb, l, r, d, n, gate);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static int boundary(const double* qb, double* fb, const int* c, const int* f, int n, int kind, const int* gate,
                      cudaStream_t st) {
    if (n <= 0) return EXA_OK;
    boundary_kernel<DIM, N, PDE><<<(n + 3) / 4, 128, 0, st>>>(qb, fb, c, f, n, kind, gate);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static int corrector(double* luh, const double* du, const double* fb, const double* dt, double* dtout, Geometry g,
                       int n, const int* list, int upd, const int* cnt, cudaStream_t st) {
    return launch_corrector<DIM, N, PDE>(luh, du, fb, dt, dtout, g, n, list, upd, cnt, st);
  }
  static KernelSet make(int pde) {
    using S = Shape<DIM, N, PDE>;
    KernelSet k{DIM, N, pde, S::nV, S::nP, S::P, S::F, false, &predictor, &riemann, &boundary, &corrector, nullptr};
    AmrLaunch<DIM, N, PDE>::fill(k);
    return k;
  }
};

// Launchers of a linear PDE (PDE::kLinear): the Cauchy-Kovalevski predictor
// with the linear volume integral, the linear Riemann solver, and the
// corrector with the linear surface integral. The predictor has one shape, so
// the variant is ignored; there are no Picard sweeps to count. Boundary
// faces: the PDE's boundaryValues and the linear Riemann solve against them.
template <int DIM, int N, class PDE>
struct LinearLaunch {
  using CC = CorrectorCfg<DIM, N, PDE>;
  using KC = CKCfg<DIM, N, PDE>;
  static_assert(KC::SMEM <= 227 * 1024, "shared memory");
  template <int NREG>
  static int launch_ck(const double* luh, double* qb, double* fb, double* du, const double* dt, Geometry g, int n,
                       const int* list, const int* cnt, double* qhi, double* fhi, cudaStream_t st) {
    static bool attr = false;
    if (!attr) {
      EXA_CUDA(cudaFuncSetAttribute(ck_predictor_kernel<DIM, N, PDE, NREG>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)KC::SMEM));
      attr = true;
    }
    ck_predictor_kernel<DIM, N, PDE, NREG><<<(n + KC::CPB - 1) / KC::CPB, KC::THREADS, KC::SMEM, st>>>(
        luh, qb, fb, du, dt, g, n, list, cnt, qhi, fhi);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  // variant 0: the register cap of one block per SM; 1: of two blocks per
  // SM (where their shared memory fits); the autotuner picks
  static constexpr bool kTwo = 2 * KC::SMEM <= 227 * 1024;
  static constexpr int kReg1 = regs_for_blocks<KC::THREADS, 1>(), kReg2 = regs_for_blocks<KC::THREADS, 2>();
  static int predictor(const double* luh, double* qb, double* fb, double* du, int*, const double* dt, Geometry g,
                       int n, const int* list, const int* cnt, PredictorTemps tmp, bool temps, unsigned long long*,
                       int variant, cudaStream_t st) {
    if (n <= 0) return EXA_OK;
    double* qhi = temps ? tmp.lQhi : nullptr;
    double* fhi = temps ? tmp.lFhi : nullptr;
    if (variant == 1 && kTwo) return launch_ck<kTwo ? kReg2 : kReg1>(luh, qb, fb, du, dt, g, n, list, cnt, qhi, fhi, st);
    return launch_ck<kReg1>(luh, qb, fb, du, dt, g, n, list, cnt, qhi, fhi, st);
  }
  static int riemann(const double* qb, double* fb, const int* l, const int* r, const int* d, int n, const int* gate,
                     cudaStream_t st) {
    if (n <= 0) return EXA_OK;
    riemann_linear_kernel<DIM, N, PDE><<<(n + 3) / 4, 128, 0, st>>>(qb, fb, l, r, d, n, gate);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static int boundary(const double* qb, double* fb, const int* c, const int* f, int n, int kind, const int* gate,
                      cudaStream_t st) {
    if (n <= 0) return EXA_OK;
    boundary_linear_kernel<DIM, N, PDE><<<(n + 3) / 4, 128, 0, st>>>(qb, fb, c, f, n, kind, gate);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static int corrector(double* luh, const double* du, const double* fb, const double* dt, double* dtout, Geometry g,
                       int n, const int* list, int upd, const int* cnt, cudaStream_t st) {
    return launch_corrector<DIM, N, PDE>(luh, du, fb, dt, dtout, g, n, list, upd, cnt, st);
  }
  static int volume(double* du, const double* fhi, int n, cudaStream_t st) {
    if (n <= 0) return EXA_OK;
    const long long total = (long long)n * Shape<DIM, N, PDE>::P;
    volume_linear_kernel<DIM, N, PDE><<<(unsigned)((total + 255) / 256), 256, 0, st>>>(du, fhi, n);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static KernelSet make(int pde) {
    using S = Shape<DIM, N, PDE>;
    KernelSet k{DIM, N, pde, S::nV, S::nP, S::P, S::F, true, &predictor, &riemann, &boundary, &corrector, &volume};
    AmrLaunch<DIM, N, PDE>::fill(k);
    k.point_source = PDE::kPointSource;
    return k;
  }
};

#define EXA_ORDERS_EULER(X, D) X(D, 3, EulerPDE, 0) X(D, 4, EulerPDE, 0) X(D, 5, EulerPDE, 0) X(D, 7, EulerPDE, 0)
#define EXA_ORDERS_TEST(X, D) X(D, 3, EulerTestPDE, 1) X(D, 5, EulerTestPDE, 1)
#define EXA_ORDERS_SOURCE_NCP(X, D) X(D, 3, EulerSourceNCPPDE, 3) X(D, 5, EulerSourceNCPPDE, 3)
#define EXA_ORDERS_ELASTIC(X, D) X(D, 3, ElasticPDE, 2) X(D, 4, ElasticPDE, 2) X(D, 5, ElasticPDE, 2)
#define EXA_ORDERS_ELASTIC_PS(X, D) X(D, 3, ElasticPointSourcePDE, 4) X(D, 5, ElasticPointSourcePDE, 4)

static bool find_kernels(int dim, int order, int pde, KernelSet* out) {
#define X(D, NN, PDE_, ID)                                     \
  if (dim == D && order == NN && pde == ID) {                 \
    *out = Launch<D, NN, PDE_>::make(ID);                     \
    return true;                                               \
  }
  EXA_ORDERS_EULER(X, 2)
  EXA_ORDERS_EULER(X, 3)
  EXA_ORDERS_TEST(X, 2)
  EXA_ORDERS_TEST(X, 3)
  EXA_ORDERS_SOURCE_NCP(X, 2)
  EXA_ORDERS_SOURCE_NCP(X, 3)
#undef X
#define X(D, NN, PDE_, ID)                                     \
  if (dim == D && order == NN && pde == ID) {                 \
    *out = LinearLaunch<D, NN, PDE_>::make(ID);               \
    return true;                                               \
  }
  EXA_ORDERS_ELASTIC(X, 2)
  EXA_ORDERS_ELASTIC(X, 3)
  EXA_ORDERS_ELASTIC_PS(X, 2)
  EXA_ORDERS_ELASTIC_PS(X, 3)
#undef X
  return false;
}

__global__ void advance_kernel(double* scal) {
  // scal: [0] dt of the current step, [1] min-reduction target, [2] time,
  //       [3] steps taken
  scal[2] += scal[0];
  scal[0] = scal[1];
  scal[1] = __longlong_as_double(0x7fefffffffffffffll);
  scal[3] += 1.0;
}

__global__ void init_scalars_kernel(double* scal, double t0) {
  scal[0] = 0.0;
  scal[1] = __longlong_as_double(0x7fefffffffffffffll);
  scal[2] = t0;
  scal[3] = 0.0;
}

__global__ void take_dt_kernel(double* scal) {
  scal[0] = scal[1];
  scal[1] = __longlong_as_double(0x7fefffffffffffffll);
}

// Refined meshes with L levels: lv[0..L-1] the step size each level's
// kernels read, lv[L..2L-1] the levels' min-reduction targets. The global
// step is the min over all levels (global time stepping).
__global__ void level_reset_kernel(double* lv, int L) {
  for (int l = 0; l < L; l++) lv[L + l] = __longlong_as_double(0x7fefffffffffffffll);
}
__device__ void level_take(double* scal, double* lv, int L) {
  double s = __longlong_as_double(0x7fefffffffffffffll);
  for (int l = 0; l < L; l++) {
    s = (lv[L + l] < s) ? lv[L + l] : s;
    lv[L + l] = __longlong_as_double(0x7fefffffffffffffll);
  }
  scal[0] = s;
  for (int l = 0; l < L; l++) lv[l] = s;
}
__global__ void level_take_kernel(double* scal, double* lv, int L) { level_take(scal, lv, L); }
__global__ void level_advance_kernel(double* scal, double* lv, int L) {
  scal[2] += scal[0];
  level_take(scal, lv, L);
  scal[3] += 1.0;
}

// validateNoNansInADERDGSolver (exahype/solvers/ADERDGSolver.cpp:1778-1829)
// as a scan: flag[cell] = 1 where any of the cell's `per_cell` values is not
// finite; then the flags are counted
__global__ void __launch_bounds__(256) nonfinite_flag_kernel(const double* __restrict__ a, size_t per_cell,
                                                             size_t total, int* __restrict__ flag) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
    if (!isfinite(a[i])) flag[i / per_cell] = 1;
}
__global__ void __launch_bounds__(256) count_flags_kernel(const int* __restrict__ flag, int n,
                                                          unsigned long long* __restrict__ count) {
  unsigned long long c = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) c += flag[i] != 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// dst cell to[k] = src cell from[k], per_cell doubles each
__global__ void __launch_bounds__(256) copy_cells_kernel(double* __restrict__ dst, const double* __restrict__ src,
                                                         size_t per_cell, int n, const int* __restrict__ to,
                                                         const int* __restrict__ from) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)n * per_cell;
       i += (size_t)gridDim.x * blockDim.x) {
    const size_t k = i / per_cell, e = i - k * per_cell;
    dst[(size_t)to[k] * per_cell + e] = src[(size_t)from[k] * per_cell + e];
  }
}

// independent FP64 FMA chains: 8 per thread, `iters` rounds
__global__ void __launch_bounds__(256) fp64_probe_kernel(double* out, int iters, double a, double b) {
  double x[8];
#pragma unroll
  for (int i = 0; i < 8; i++) x[i] = threadIdx.x * 1e-3 + i;
  for (int k = 0; k < iters; k++) {
#pragma unroll
    for (int i = 0; i < 8; i++) x[i] = fma(x[i], a, b);
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) s += x[i];
  if (s == 1.2345e300) out[0] = s;  // never true; keeps the chains alive
}

// FP64 tensor-core (DMMA) throughput: 4 independent m8n8k4 accumulator chains
// per warp, `iters` rounds; 2 * 256 flops per warp and MMA
__global__ void __launch_bounds__(256) fp64_mma_probe_kernel(double* out, int iters, double a, double b) {
  double d[4][2];
#pragma unroll
  for (int i = 0; i < 4; i++) d[i][0] = d[i][1] = threadIdx.x * 1e-3 + i;
  for (int k = 0; k < iters; k++) {
#pragma unroll
    for (int i = 0; i < 4; i++)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(d[i][0]), "+d"(d[i][1])
                   : "d"(a), "d"(b));
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < 4; i++) s += d[i][0] + d[i][1];
  if (s == 1.2345e300) out[0] = s;  // never true; keeps the chains alive
}

}  // namespace exa

using namespace exa;

struct exa_solver {
  KernelSet k;
  int variant = 0;  // predictor variant (set by exa_solver_autotune / exa_solver_set_variant)
  // point source of a PDE with one (exa_solver_set_point_source): position
  // x0[3], delay t0, peak frequency f0, amplitude
  double ps[6] = {0.5, 0.5, 0.5, 0.1, 8.0, 1.0};
};

// one level of a refined mesh on the host: the bounding rectangle [r0, r1)
// of its region, per position 0 outside / 1 cell / 2 refined, and the cell
// index (or -1)
struct LevelMap {
  std::array<int, 3> r0{}, r1{};
  std::vector<unsigned char> st;
  std::vector<int> cell;
  bool inside(const int* p) const {
    for (int d = 0; d < 3; d++)
      if (p[d] < r0[d] || p[d] >= r1[d]) return false;
    return true;
  }
  size_t at(const int* p) const {
    return ((size_t)(p[2] - r0[2]) * (r1[1] - r0[1]) + (p[1] - r0[1])) * (r1[0] - r0[0]) + (p[0] - r0[0]);
  }
};

struct exa_mesh {
  const exa_solver* s = nullptr;
  int dim = 0, cells[3] = {1, 1, 1}, ncells = 0, bc[6] = {0, 0, 0, 0, 0, 0};
  Geometry geo{};
  double offset[3] = {0, 0, 0}, size[3] = {1, 1, 1};
  double *luh = nullptr, *lduh = nullptr, *lQhbnd = nullptr, *lFhbnd = nullptr, *scal = nullptr;
  int *iters = nullptr, *fl = nullptr, *fr = nullptr, *fd = nullptr, *bcell = nullptr, *bface = nullptr;
  int nfaces = 0, nbfaces[3] = {0, 0, 0};  // boundary faces grouped by kind: outflow, reflective
  int boff[3] = {0, 0, 0};
  unsigned long long* sweeps = nullptr;
  double* centre = nullptr;  // cell centres [cell][3] (point-source PDEs only)
  cudaStream_t stream = nullptr;
  bool initialised = false;
  // optional per-phase event timing
  bool profiling = false;
  std::vector<cudaEvent_t> ev;   // pairs (start, stop) recorded, not yet folded in
  std::vector<int> ev_phase;
  double phase_ms[4] = {0, 0, 0, 0};
  long long phase_launches[4] = {0, 0, 0, 0};
  // streamed host I/O of exa_mesh_step_io: staging buffers, copy streams and
  // the events that order them against the mesh stream
  double *stage_in = nullptr, *stage_out = nullptr;
  cudaStream_t io_in = nullptr, io_out = nullptr;
  cudaEvent_t in_ready = nullptr, in_free = nullptr, out_ready = nullptr, out_free = nullptr;
  // fused time stepping (exa_mesh_init_fused): rerun weight and the device
  // count of cells whose predictor is rerun (0 or all)
  bool fused = false;
  double weight = 0.99;
  int* rerun = nullptr;
  // statically refined mesh (exa_mesh_create_nested / _refined): nlev
  // levels as geometry instances (per-cell level index, per-level widths),
  // per-level step sizes and min-reduction targets lv[0..nlev-1],
  // lv[nlev..2 nlev-1], the face slots of the refined cells that face
  // coarser cells (ancestors, zeroed and restricted into after every
  // predictor) and of the virtual finer cells across each refined box's
  // faces (descendants, prolongated into)
  struct {
    bool on = false;
    int nlev = 1;
    double* lv = nullptr;
    int* inst = nullptr;
    double* inst_dx = nullptr;
    int anc0 = 0, nanc = 0, nres = 0, npro = 0;
    int *res_f = nullptr, *res_c = nullptr, *res_ld = nullptr, *res_idx = nullptr;
    int *pro_f = nullptr, *pro_c = nullptr, *pro_ld = nullptr, *pro_idx = nullptr;
    // host copies for the VTK writers: each cell's level and grid position,
    // each level's widths
    std::vector<int> level, pos;
    std::vector<double> ldx;
    std::vector<LevelMap> maps;  // per level (for exa_mesh_regrid)
  } ref;
};

namespace {
struct PhaseTimer {
  exa_mesh* m;
  int phase;
  cudaEvent_t a = nullptr, b = nullptr;
  PhaseTimer(exa_mesh* mm, int ph) : m(mm), phase(ph) {
    if (!m->profiling) return;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, m->stream);
  }
  ~PhaseTimer() {
    if (!m->profiling) return;
    cudaEventRecord(b, m->stream);
    m->ev.push_back(a);
    m->ev.push_back(b);
    m->ev_phase.push_back(phase);
  }
};
}  // namespace

extern "C" {

const char* exa_last_error(void) { return g_last_error.c_str(); }
const char* exa_version(void) { return "exahype_b200 0.1 (sm_100a, FP64 ADER-DG)"; }

int exa_solver_create(int dim, int order, int pde, exa_solver** out) {
  if (!out) return fail(EXA_ERR_ARG, "exa_solver_create: out is NULL");
  if (dim != 2 && dim != 3) return fail(EXA_ERR_ARG, "exa_solver_create: dim must be 2 or 3");
  if (order < 1 || order > kMaxOrder) return fail(EXA_ERR_ARG, "exa_solver_create: order out of range 1..9");
  KernelSet k{};
  if (!find_kernels(dim, order, pde, &k))
    return fail(EXA_ERR_UNSUPPORTED, "exa_solver_create: no kernels built for dim=" + std::to_string(dim) +
                                         " order=" + std::to_string(order) + " pde=" + std::to_string(pde));
  int rc = upload_tables();
  if (rc) return rc;
  *out = new exa_solver{k};
  return EXA_OK;
}

int exa_solver_destroy(exa_solver* s) {
  delete s;
  return EXA_OK;
}

int exa_solver_sizes(const exa_solver* s, int* z) {
  if (!s || !z) return fail(EXA_ERR_ARG, "exa_solver_sizes: null argument");
  z[0] = s->k.P * s->k.nvar;
  z[1] = s->k.P * (s->k.nvar + s->k.npar);
  z[2] = s->k.F * (s->k.nvar + s->k.npar);
  z[3] = s->k.F * s->k.nvar;
  return EXA_OK;
}

static Geometry geom(const exa_solver* s, const double* dx) {
  Geometry g{};
  for (int d = 0; d < 3; d++) g.dx[d] = d < s->k.dim ? dx[d] : 1.0;
  for (int i = 0; i < 6; i++) g.ps[i] = s->ps[i];
  return g;
}

int exa_solver_set_point_source(exa_solver* s, const double* x0, double t0, double f0, double amplitude) {
  if (!s || !x0) return fail(EXA_ERR_ARG, "exa_solver_set_point_source: null argument");
  if (!s->k.point_source) return fail(EXA_ERR_UNSUPPORTED, "exa_solver_set_point_source: the PDE has no point source");
  if (!std::isfinite(t0) || !std::isfinite(f0) || !std::isfinite(amplitude))
    return fail(EXA_ERR_ARG, "exa_solver_set_point_source: non-finite parameter");
  for (int d = 0; d < 3; d++) s->ps[d] = d < s->k.dim ? x0[d] : 0.0;
  s->ps[3] = t0;
  s->ps[4] = f0;
  s->ps[5] = amplitude;
  return EXA_OK;
}

int exa_space_time_predictor_nonlinear(const exa_solver* s, const double* luh, double* lQhbnd, double* lFhbnd,
                                       double* lduh, const double* dt_dev, const double* dx, int ncells,
                                       const int* cell_list, int* iterations_dev, void* stream) {
  if (!s || !luh || !lQhbnd || !lFhbnd || !dt_dev || !dx || ncells < 0)
    return fail(EXA_ERR_ARG, "exa_space_time_predictor_nonlinear: null argument or negative count");
  if (s->k.linear) return fail(EXA_ERR_UNSUPPORTED, "exa_space_time_predictor_nonlinear: linear PDE, use _linear");
  return s->k.predictor(luh, lQhbnd, lFhbnd, lduh, iterations_dev, dt_dev, geom(s, dx), ncells, cell_list, nullptr,
                        PredictorTemps{}, false, nullptr, s->variant, (cudaStream_t)stream);
}

int exa_space_time_predictor_nonlinear_temps(const exa_solver* s, const double* luh, double* lQhbnd,
                                             double* lFhbnd, double* lduh, const double* dt_dev, const double* dx,
                                             int ncells, int* iterations_dev, double* lQi, double* lFi,
                                             double* lQhi, double* lFhi, void* stream) {
  if (!s || !luh || !lQhbnd || !lFhbnd || !dt_dev || !dx || ncells < 0 || !lQi || !lFi || !lQhi || !lFhi)
    return fail(EXA_ERR_ARG, "exa_space_time_predictor_nonlinear_temps: null argument or negative count");
  if (s->k.linear)
    return fail(EXA_ERR_UNSUPPORTED, "exa_space_time_predictor_nonlinear_temps: linear PDE, use _linear_temps");
  return s->k.predictor(luh, lQhbnd, lFhbnd, lduh, iterations_dev, dt_dev, geom(s, dx), ncells, nullptr, nullptr,
                        PredictorTemps{lQi, lFi, lQhi, lFhi}, true, nullptr, s->variant, (cudaStream_t)stream);
}

int exa_riemann_solver_nonlinear(const exa_solver* s, const double* lQhbnd, double* lFhbnd, const int* face_left,
                                 const int* face_right, const int* face_dir, int nfaces, void* stream) {
  if (!s || !lQhbnd || !lFhbnd || nfaces < 0 || (nfaces > 0 && (!face_left || !face_right || !face_dir)))
    return fail(EXA_ERR_ARG, "exa_riemann_solver_nonlinear: null argument or negative count");
  if (s->k.linear) return fail(EXA_ERR_UNSUPPORTED, "exa_riemann_solver_nonlinear: linear PDE, use _linear");
  return s->k.riemann(lQhbnd, lFhbnd, face_left, face_right, face_dir, nfaces, nullptr, (cudaStream_t)stream);
}

int exa_space_time_predictor_linear(const exa_solver* s, const double* luh, double* lQhbnd, double* lFhbnd,
                                    double* lduh, const double* dt_dev, const double* dx, int ncells,
                                    const int* cell_list, void* stream) {
  if (!s || !luh || !lQhbnd || !lFhbnd || !dt_dev || !dx || ncells < 0)
    return fail(EXA_ERR_ARG, "exa_space_time_predictor_linear: null argument or negative count");
  if (!s->k.linear) return fail(EXA_ERR_UNSUPPORTED, "exa_space_time_predictor_linear: nonlinear PDE");
  if (s->k.point_source)
    return fail(EXA_ERR_UNSUPPORTED, "exa_space_time_predictor_linear: point-source PDE, use _linear_point_source");
  return s->k.predictor(luh, lQhbnd, lFhbnd, lduh, nullptr, dt_dev, geom(s, dx), ncells, cell_list, nullptr,
                        PredictorTemps{}, false, nullptr, s->variant, (cudaStream_t)stream);
}

int exa_space_time_predictor_linear_point_source(const exa_solver* s, const double* luh, double* lQhbnd,
                                                 double* lFhbnd, double* lduh, const double* t_dev,
                                                 const double* dt_dev, const double* dx, const double* centres,
                                                 int ncells, const int* cell_list, double* lQhi, double* lFhi,
                                                 void* stream) {
  if (!s || !luh || !lQhbnd || !lFhbnd || !t_dev || !dt_dev || !dx || !centres || ncells < 0 || (!lQhi != !lFhi))
    return fail(EXA_ERR_ARG, "exa_space_time_predictor_linear_point_source: null argument or negative count");
  if (!s->k.linear || !s->k.point_source)
    return fail(EXA_ERR_UNSUPPORTED, "exa_space_time_predictor_linear_point_source: the PDE has no point source");
  Geometry g = geom(s, dx);
  g.centre = centres;
  g.time = t_dev;
  const bool temps = lQhi != nullptr;
  return s->k.predictor(luh, lQhbnd, lFhbnd, lduh, nullptr, dt_dev, g, ncells, cell_list, nullptr,
                        PredictorTemps{nullptr, nullptr, lQhi, lFhi}, temps, nullptr, s->variant,
                        (cudaStream_t)stream);
}

int exa_space_time_predictor_linear_temps(const exa_solver* s, const double* luh, double* lQhbnd, double* lFhbnd,
                                          double* lduh, const double* dt_dev, const double* dx, int ncells,
                                          double* lQhi, double* lFhi, void* stream) {
  if (!s || !luh || !lQhbnd || !lFhbnd || !dt_dev || !dx || ncells < 0 || !lQhi || !lFhi)
    return fail(EXA_ERR_ARG, "exa_space_time_predictor_linear_temps: null argument or negative count");
  if (!s->k.linear) return fail(EXA_ERR_UNSUPPORTED, "exa_space_time_predictor_linear_temps: nonlinear PDE");
  if (s->k.point_source)
    return fail(EXA_ERR_UNSUPPORTED, "exa_space_time_predictor_linear_temps: point-source PDE, use _linear_point_source");
  return s->k.predictor(luh, lQhbnd, lFhbnd, lduh, nullptr, dt_dev, geom(s, dx), ncells, nullptr, nullptr,
                        PredictorTemps{nullptr, nullptr, lQhi, lFhi}, true, nullptr, s->variant,
                        (cudaStream_t)stream);
}

int exa_riemann_solver_linear(const exa_solver* s, const double* lQhbnd, double* lFhbnd, const int* face_left,
                              const int* face_right, const int* face_dir, int nfaces, void* stream) {
  if (!s || !lQhbnd || !lFhbnd || nfaces < 0 || (nfaces > 0 && (!face_left || !face_right || !face_dir)))
    return fail(EXA_ERR_ARG, "exa_riemann_solver_linear: null argument or negative count");
  if (!s->k.linear) return fail(EXA_ERR_UNSUPPORTED, "exa_riemann_solver_linear: nonlinear PDE");
  return s->k.riemann(lQhbnd, lFhbnd, face_left, face_right, face_dir, nfaces, nullptr, (cudaStream_t)stream);
}

int exa_volume_integral_linear(const exa_solver* s, double* lduh, const double* lFhi, int ncells, void* stream) {
  if (!s || !lduh || !lFhi || ncells < 0)
    return fail(EXA_ERR_ARG, "exa_volume_integral_linear: null argument or negative count");
  if (!s->k.linear) return fail(EXA_ERR_UNSUPPORTED, "exa_volume_integral_linear: nonlinear PDE");
  return s->k.volume(lduh, lFhi, ncells, (cudaStream_t)stream);
}

int exa_volume_unknowns_prolongation(const exa_solver* s, double* luh_fine, const double* luh_coarse, int n,
                                     const int* fine_cell, const int* coarse_cell, const int* level_delta,
                                     const int* subcell_index, void* stream) {
  if (!s || !luh_fine || !luh_coarse || n < 0 ||
      (n > 0 && (!fine_cell || !coarse_cell || !level_delta || !subcell_index)))
    return fail(EXA_ERR_ARG, "exa_volume_unknowns_prolongation: null argument or negative count");
  return s->k.amr_volume(luh_fine, luh_coarse, n, fine_cell, coarse_cell, level_delta, subcell_index, 0,
                         (cudaStream_t)stream);
}

int exa_volume_unknowns_restriction(const exa_solver* s, double* luh_coarse, const double* luh_fine, int n,
                                    const int* fine_cell, const int* coarse_cell, const int* level_delta,
                                    const int* subcell_index, void* stream) {
  if (!s || !luh_fine || !luh_coarse || n < 0 ||
      (n > 0 && (!fine_cell || !coarse_cell || !level_delta || !subcell_index)))
    return fail(EXA_ERR_ARG, "exa_volume_unknowns_restriction: null argument or negative count");
  return s->k.amr_volume(luh_coarse, luh_fine, n, fine_cell, coarse_cell, level_delta, subcell_index, 1,
                         (cudaStream_t)stream);
}

int exa_face_unknowns_prolongation(const exa_solver* s, double* lQhbnd_fine, double* lFhbnd_fine,
                                   const double* lQhbnd_coarse, const double* lFhbnd_coarse, int n,
                                   const int* fine_slot, const int* coarse_slot, const int* level_delta,
                                   const int* subface_index, void* stream) {
  if (!s || !lQhbnd_fine || !lFhbnd_fine || !lQhbnd_coarse || !lFhbnd_coarse || n < 0 ||
      (n > 0 && (!fine_slot || !coarse_slot || !level_delta || !subface_index)))
    return fail(EXA_ERR_ARG, "exa_face_unknowns_prolongation: null argument or negative count");
  return s->k.amr_face(lQhbnd_fine, lFhbnd_fine, lQhbnd_coarse, lFhbnd_coarse, n, fine_slot, coarse_slot,
                       level_delta, subface_index, 0, (cudaStream_t)stream);
}

int exa_face_unknowns_restriction(const exa_solver* s, double* lQhbnd_coarse, double* lFhbnd_coarse,
                                  const double* lQhbnd_fine, const double* lFhbnd_fine, int n, const int* fine_slot,
                                  const int* coarse_slot, const int* level_delta, const int* subface_index,
                                  void* stream) {
  if (!s || !lQhbnd_fine || !lFhbnd_fine || !lQhbnd_coarse || !lFhbnd_coarse || n < 0 ||
      (n > 0 && (!fine_slot || !coarse_slot || !level_delta || !subface_index)))
    return fail(EXA_ERR_ARG, "exa_face_unknowns_restriction: null argument or negative count");
  return s->k.amr_face(lQhbnd_coarse, lFhbnd_coarse, lQhbnd_fine, lFhbnd_fine, n, fine_slot, coarse_slot,
                       level_delta, subface_index, 1, (cudaStream_t)stream);
}

int exa_plot_vertices(const exa_solver* s, const double* luh, double* vertices, int ncells, void* stream) {
  if (!s || !luh || !vertices || ncells < 0)
    return fail(EXA_ERR_ARG, "exa_plot_vertices: null argument or negative count");
  return s->k.plot(luh, vertices, ncells, (cudaStream_t)stream);
}

int exa_boundary_conditions(const exa_solver* s, const double* lQhbnd, double* lFhbnd, const int* bcell,
                            const int* bface, int nb, int kind, void* stream) {
  if (!s || !lQhbnd || !lFhbnd || nb < 0 || (nb > 0 && (!bcell || !bface)))
    return fail(EXA_ERR_ARG, "exa_boundary_conditions: null argument or negative count");
  if (kind != EXA_BC_OUTFLOW && kind != EXA_BC_REFLECTIVE)
    return fail(EXA_ERR_ARG, "exa_boundary_conditions: kind must be outflow or reflective");
  return s->k.boundary(lQhbnd, lFhbnd, bcell, bface, nb, kind, nullptr, (cudaStream_t)stream);
}

int exa_corrector(const exa_solver* s, double* luh, const double* lduh, const double* lFhbnd, const double* dt_dev,
                  double* dt_min_dev, const double* dx, int ncells, const int* cell_list, int update, void* stream) {
  if (!s || !luh || !dx || ncells < 0 || (update && (!lduh || !lFhbnd || !dt_dev)))
    return fail(EXA_ERR_ARG, "exa_corrector: null argument or negative count");
  return s->k.corrector(luh, lduh, lFhbnd, dt_dev, dt_min_dev, geom(s, dx), ncells, cell_list, update, nullptr,
                        (cudaStream_t)stream);
}

int exa_reset_min(double* dev, void* stream) {
  if (!dev) return fail(EXA_ERR_ARG, "exa_reset_min: null pointer");
  reset_min_kernel<<<1, 1, 0, (cudaStream_t)stream>>>(dev);
  EXA_LAUNCHED();
  return EXA_OK;
}

// smooth synthetic states for the autotuner: rho, j, E with O(10%) variation
// (parameters, v >= nV, positive: the elastic PDE divides by rho)
__global__ void autotune_fill_kernel(double* luh, long long n, int nD, int nV) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long node = i / nD;
    const int v = (int)(i - node * nD);
    const double s = sin(0.37 * (double)node) * cos(0.011 * (double)node);
    luh[i] = v >= nV ? 1.5 + 0.2 * s : v == 0 ? 1.0 + 0.1 * s : v == 4 ? 2.5 + 0.2 * s : v < 4 ? 0.3 * s * (v - 2) : 0.0;
  }
}

int exa_solver_set_variant(exa_solver* s, int variant) {
  if (!s || variant < 0 || variant >= kAllVariants) return fail(EXA_ERR_ARG, "exa_solver_set_variant: bad argument");
  s->variant = variant;
  return EXA_OK;
}

int exa_solver_get_variant(const exa_solver* s, int* variant) {
  if (!s || !variant) return fail(EXA_ERR_ARG, "exa_solver_get_variant: null argument");
  *variant = s->variant;
  return EXA_OK;
}

int exa_solver_autotune(exa_solver* s, int ncells, double* variant_ms, int* chosen) {
  if (!s || ncells < 1) return fail(EXA_ERR_ARG, "exa_solver_autotune: bad argument");
  const KernelSet& k = s->k;
  const size_t P = k.P, F = k.F, nV = k.nvar, nD = k.nvar + k.npar, D2 = 2 * k.dim, n = ncells;
  double *luh = nullptr, *qb = nullptr, *fb = nullptr, *du = nullptr, *dt = nullptr;
  int* it = nullptr;
  auto cleanup = [&]() { cudaFree(luh); cudaFree(qb); cudaFree(fb); cudaFree(du); cudaFree(dt); cudaFree(it); };
  if (cudaMalloc(&luh, n * P * nD * 8) != cudaSuccess || cudaMalloc(&qb, n * D2 * F * nD * 8) != cudaSuccess ||
      cudaMalloc(&fb, n * D2 * F * nV * 8) != cudaSuccess || cudaMalloc(&du, n * P * nV * 8) != cudaSuccess ||
      cudaMalloc(&dt, 8) != cudaSuccess || cudaMalloc(&it, n * 4) != cudaSuccess) {
    cudaGetLastError();
    cleanup();
    return fail(EXA_ERR_NOMEM, "exa_solver_autotune: device allocation failed");
  }
  cudaStream_t st;
  EXA_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  autotune_fill_kernel<<<1024, 256, 0, st>>>(luh, (long long)(n * P * nD), (int)nD, (int)nV);
  Geometry g{};
  for (int d = 0; d < 3; d++) g.dx[d] = 1.0 / 27.0;
  reset_min_kernel<<<1, 1, 0, st>>>(dt);
  int rc = k.corrector(luh, nullptr, nullptr, nullptr, dt, g, (int)n, nullptr, 0, nullptr, st);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  int best = 0;
  double best_ms = 1e300;
  for (int v = 0; v < kAllVariants && rc == EXA_OK; v++) {
    if (variant_is_mixed(v) || (k.linear && v > 1)) {  // mixed: changes the results; linear: two shapes
      if (variant_ms) variant_ms[v] = -1.0;
      continue;
    }
    float ms = 0.f, tot = 0.f;
    for (int r = 0; r < 4 && rc == EXA_OK; r++) {
      cudaEventRecord(a, st);
      rc = k.predictor(luh, qb, fb, du, it, dt, g, (int)n, nullptr, nullptr, PredictorTemps{}, false, nullptr, v, st);
      cudaEventRecord(b, st);
      cudaEventSynchronize(b);
      cudaEventElapsedTime(&ms, a, b);
      if (r > 0) tot += ms;  // first launch is a warm-up
    }
    const double avg = tot / 3.0;
    if (variant_ms) variant_ms[v] = avg;
    if (avg < best_ms) {
      best_ms = avg;
      best = v;
    }
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  cleanup();
  if (rc) return rc;
  s->variant = best;
  if (chosen) *chosen = best;
  return EXA_OK;
}

// ---- mesh -------------------------------------------------------------------
static void mesh_free(exa_mesh* m) {
  for (cudaEvent_t e : m->ev) cudaEventDestroy(e);
  m->ev.clear();
  if (m->io_in) cudaStreamSynchronize(m->io_in);
  if (m->io_out) cudaStreamSynchronize(m->io_out);
  for (cudaEvent_t e : {m->in_ready, m->in_free, m->out_ready, m->out_free})
    if (e) cudaEventDestroy(e);
  sfree(m->stage_in, m->stream);
  sfree(m->stage_out, m->stream);
  sfree(m->rerun, m->stream);
  for (void* p : {(void*)m->ref.lv, (void*)m->ref.inst, (void*)m->ref.inst_dx, (void*)m->ref.res_f,
                  (void*)m->ref.res_c, (void*)m->ref.res_ld, (void*)m->ref.res_idx, (void*)m->ref.pro_f,
                  (void*)m->ref.pro_c, (void*)m->ref.pro_ld, (void*)m->ref.pro_idx})
    sfree(p, m->stream);
  if (m->io_in) cudaStreamDestroy(m->io_in);
  if (m->io_out) cudaStreamDestroy(m->io_out);
  for (void* p : {(void*)m->luh, (void*)m->lduh, (void*)m->lQhbnd, (void*)m->lFhbnd, (void*)m->scal, (void*)m->iters,
                  (void*)m->fl, (void*)m->fr, (void*)m->fd, (void*)m->bcell, (void*)m->bface, (void*)m->sweeps,
                  (void*)m->centre})
    sfree(p, m->stream);
  if (m->stream) cudaStreamDestroy(m->stream);
}

// Cell centres of a point-source PDE's mesh: cell c at grid position p of a
// level of widths h spans [offset + p h, offset + (p + 1) h]; its centre is
// offset + p h + h / 2 (the cell offset plus half its size, as the reference
// passes it to pointSource, ADERDGSolver.cpp:1929). pos: 3 ints per cell;
// widths: 3 doubles per level (level per cell, or all 0).
static int mesh_centres(exa_mesh* m, const std::vector<int>& pos, const std::vector<int>* level,
                        const std::vector<double>& widths) {
  if (!m->s->k.point_source) return EXA_OK;
  std::vector<double> c(3 * (size_t)m->ncells, 0.0);
  for (size_t i = 0; i < (size_t)m->ncells; i++) {
    const double* h = &widths[3 * (size_t)(level ? (*level)[i] : 0)];
    for (int d = 0; d < m->dim; d++) c[3 * i + d] = (m->offset[d] + pos[3 * i + d] * h[d]) + 0.5 * h[d];
  }
  if (!salloc(&m->centre, c.size() * 8, m->stream)) {
    cudaGetLastError();
    m->centre = nullptr;
    return fail(EXA_ERR_NOMEM, "mesh: device allocation of the cell centres failed");
  }
  EXA_CUDA(cudaMemcpyAsync(m->centre, c.data(), c.size() * 8, cudaMemcpyHostToDevice, m->stream));
  EXA_CUDA(cudaStreamSynchronize(m->stream));  // c goes out of scope
  m->geo.centre = m->centre;
  return EXA_OK;
}

int exa_mesh_create(const exa_solver* s, const int* cells, const double* offset, const double* size, const int* bc,
                    exa_mesh** out) {
  if (!s || !cells || !offset || !size || !bc || !out) return fail(EXA_ERR_ARG, "exa_mesh_create: null argument");
  std::unique_ptr<exa_mesh> m(new exa_mesh());
  m->s = s;
  m->dim = s->k.dim;
  long long nc = 1;
  for (int d = 0; d < m->dim; d++) {
    if (cells[d] < 1) return fail(EXA_ERR_ARG, "exa_mesh_create: cells per axis must be >= 1");
    if (!(size[d] > 0)) return fail(EXA_ERR_ARG, "exa_mesh_create: domain size must be > 0");
    m->cells[d] = cells[d];
    m->offset[d] = offset[d];
    m->geo.dx[d] = size[d] / cells[d];
    nc *= cells[d];
    const bool pl = bc[2 * d] == EXA_BC_PERIODIC, pr = bc[2 * d + 1] == EXA_BC_PERIODIC;
    if (pl != pr) return fail(EXA_ERR_ARG, "exa_mesh_create: periodic must be set on both faces of an axis");
    for (int f = 0; f < 2; f++) {
      const int k = bc[2 * d + f];
      if (k != EXA_BC_PERIODIC && k != EXA_BC_OUTFLOW && k != EXA_BC_REFLECTIVE)
        return fail(EXA_ERR_ARG, "exa_mesh_create: unknown boundary kind");
      m->bc[2 * d + f] = k;
    }
  }
  for (int d = m->dim; d < 3; d++) m->geo.dx[d] = 1.0;
  if (nc > (1ll << 30)) return fail(EXA_ERR_ARG, "exa_mesh_create: too many cells");
  m->ncells = (int)nc;
  // face lists: interior (incl. periodic wrap) faces per direction; boundary faces grouped by kind
  std::vector<int> fl, fr, fd, bcl[2], bfc[2];
  auto cid = [&](int i, int j, int k) { return (k * m->cells[1] + j) * m->cells[0] + i; };
  for (int k = 0; k < (m->dim == 3 ? m->cells[2] : 1); k++)
    for (int j = 0; j < m->cells[1]; j++)
      for (int i = 0; i < m->cells[0]; i++) {
        const int c = cid(i, j, k);
        int ijk[3] = {i, j, k};
        for (int d = 0; d < m->dim; d++) {
          int nb[3] = {i, j, k};
          nb[d] = ijk[d] + 1;
          if (nb[d] < m->cells[d]) {
            fl.push_back(c);
            fr.push_back(cid(nb[0], nb[1], nb[2]));
            fd.push_back(d);
          } else if (m->bc[2 * d + 1] == EXA_BC_PERIODIC) {
            nb[d] = 0;
            fl.push_back(c);
            fr.push_back(cid(nb[0], nb[1], nb[2]));
            fd.push_back(d);
          } else {
            bcl[m->bc[2 * d + 1]].push_back(c);
            bfc[m->bc[2 * d + 1]].push_back(2 * d + 1);
          }
          if (ijk[d] == 0 && m->bc[2 * d] != EXA_BC_PERIODIC) {
            bcl[m->bc[2 * d]].push_back(c);
            bfc[m->bc[2 * d]].push_back(2 * d);
          }
        }
      }
  m->nfaces = (int)fl.size();
  std::vector<int> bcell, bface;
  for (int kd = 0; kd < 2; kd++) {
    m->boff[kd] = (int)bcell.size();
    m->nbfaces[kd] = (int)bcl[kd].size();
    bcell.insert(bcell.end(), bcl[kd].begin(), bcl[kd].end());
    bface.insert(bface.end(), bfc[kd].begin(), bfc[kd].end());
  }
  const size_t P = s->k.P, F = s->k.F, nV = s->k.nvar, nD = s->k.nvar + s->k.npar, D2 = 2 * m->dim;
  const size_t n = m->ncells;
  EXA_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  cudaStream_t st = m->stream;
  bool ok = salloc(&m->luh, n * P * nD * 8, st) && salloc(&m->lduh, n * P * nV * 8, st) &&
            salloc(&m->lQhbnd, n * D2 * F * nD * 8, st) && salloc(&m->lFhbnd, n * D2 * F * nV * 8, st) &&
            salloc(&m->scal, 8 * 8, st) && salloc(&m->iters, n * 4, st) &&
            salloc(&m->fl, std::max<size_t>(1, fl.size()) * 4, st) && salloc(&m->fr, std::max<size_t>(1, fl.size()) * 4, st) &&
            salloc(&m->fd, std::max<size_t>(1, fl.size()) * 4, st) &&
            salloc(&m->bcell, std::max<size_t>(1, bcell.size()) * 4, st) &&
            salloc(&m->bface, std::max<size_t>(1, bcell.size()) * 4, st) && salloc(&m->sweeps, 8, st);
  if (!ok) {
    cudaGetLastError();
    mesh_free(m.get());
    return fail(EXA_ERR_NOMEM, "exa_mesh_create: device allocation failed");
  }
  if (!fl.empty()) {
    EXA_CUDA(cudaMemcpyAsync(m->fl, fl.data(), fl.size() * 4, cudaMemcpyHostToDevice, st));
    EXA_CUDA(cudaMemcpyAsync(m->fr, fr.data(), fr.size() * 4, cudaMemcpyHostToDevice, st));
    EXA_CUDA(cudaMemcpyAsync(m->fd, fd.data(), fd.size() * 4, cudaMemcpyHostToDevice, st));
  }
  if (!bcell.empty()) {
    EXA_CUDA(cudaMemcpyAsync(m->bcell, bcell.data(), bcell.size() * 4, cudaMemcpyHostToDevice, st));
    EXA_CUDA(cudaMemcpyAsync(m->bface, bface.data(), bface.size() * 4, cudaMemcpyHostToDevice, st));
  }
  EXA_CUDA(cudaMemsetAsync(m->luh, 0, n * P * nD * 8, st));
  EXA_CUDA(cudaMemsetAsync(m->lduh, 0, n * P * nV * 8, st));
  EXA_CUDA(cudaMemsetAsync(m->lQhbnd, 0, n * D2 * F * nD * 8, st));
  EXA_CUDA(cudaMemsetAsync(m->lFhbnd, 0, n * D2 * F * nV * 8, st));
  EXA_CUDA(cudaMemsetAsync(m->sweeps, 0, 8, st));
  EXA_CUDA(cudaStreamSynchronize(st));
  if (s->k.point_source) {
    std::vector<int> pos(3 * n, 0);
    for (size_t c = 0; c < n; c++) {
      pos[3 * c] = (int)(c % m->cells[0]);
      pos[3 * c + 1] = (int)((c / m->cells[0]) % m->cells[1]);
      pos[3 * c + 2] = (int)(c / ((size_t)m->cells[0] * m->cells[1]));
    }
    const std::vector<double> w(m->geo.dx, m->geo.dx + 3);
    if (int rc = mesh_centres(m.get(), pos, nullptr, w)) {
      mesh_free(m.get());
      return rc;
    }
  }
  *out = m.release();
  return EXA_OK;
}

// Topology of a nested refined mesh: level 0 is the periodic grid, level l
// >= 1 the box box[l-1] of level l-1 (in level-(l-1) cell coordinates)
// refined once. Slots: the cells of every level (level by level, x fastest,
// refined positions skipped), then the ancestors (refined positions on their
// box's faces), then the descendants (one per cell on a refined box's face
// and face it lies on).
namespace {
struct NestedTopo {
  int dim = 0, L = 1, ncells = 0, anc0 = 0, nanc = 0, nslots = 0;
  std::vector<int> level;                              // per cell
  std::vector<int> pos;                                // per cell: position in its level's grid (3 ints)
  std::vector<int> fl, fr, fd;                          // Riemann pairs
  std::vector<int> bcell, bface, bkind;                 // domain faces of level-0 cells and their kinds
  std::vector<int> rf, rc, ridx, pf, pc, pidx;          // restriction / prolongation items
  std::vector<LevelMap> maps;                           // per level
};

// A refined mesh from boxes: box k refines the positions lo_k <= p < hi_k
// of level box_level[k] (in that level's cell coordinates over the whole
// domain: 3^l cells[d] per axis at level l). The region of level l >= 1 is
// the union of the level-(l-1) boxes, refined once; every box must lie
// inside its level's region with one cell of margin, so that hanging faces
// join neighbouring levels only. Returns an error message, or nullptr.
static const char* boxes_topology(int dim, const int* cells, const int* bc, int nb, const int* box_level,
                                  const int* lo, const int* hi, NestedTopo& t) {
  int L = 1;
  for (int k = 0; k < nb; k++) {
    if (box_level[k] < 0 || box_level[k] > 7) return "box levels must be 0..7";
    L = std::max(L, box_level[k] + 2);
  }
  const int D2 = 2 * dim;
  t.dim = dim;
  t.L = L;
  // bounding rectangle [r0, r1) of every level's region
  std::vector<std::array<int, 3>> r0(L), r1(L);
  for (int d = 0; d < 3; d++) r0[0][d] = 0, r1[0][d] = d < dim ? cells[d] : 1;
  for (int l = 1; l < L; l++) {
    bool any = false;
    for (int d = 0; d < 3; d++) r0[l][d] = INT_MAX, r1[l][d] = INT_MIN;
    for (int k = 0; k < nb; k++) {
      if (box_level[k] != l - 1) continue;
      any = true;
      for (int d = 0; d < 3; d++) {
        const int a = d < dim ? 3 * lo[3 * k + d] : 0, b = d < dim ? 3 * hi[3 * k + d] : 1;
        r0[l][d] = std::min(r0[l][d], a);
        r1[l][d] = std::max(r1[l][d], b);
      }
    }
    if (!any) return "every level below the finest needs at least one box";
  }
  auto ext = [&](int l, int d) { return r1[l][d] - r0[l][d]; };
  for (int l = 0; l < L; l++)
    if ((double)ext(l, 0) * ext(l, 1) * ext(l, 2) > (double)(1ll << 27)) return "too many cells";
  auto inrect = [&](int l, const int* p) {
    for (int d = 0; d < 3; d++)
      if (p[d] < r0[l][d] || p[d] >= r1[l][d]) return false;
    return true;
  };
  auto idx = [&](int l, const int* p) {
    return ((size_t)(p[2] - r0[l][2]) * ext(l, 1) + (p[1] - r0[l][1])) * ext(l, 0) + (p[0] - r0[l][0]);
  };
  // state per level and position: 0 outside the region, 1 cell, 2 refined
  std::vector<std::vector<unsigned char>> st(L);
  for (int l = 0; l < L; l++) st[l].assign((size_t)ext(l, 0) * ext(l, 1) * ext(l, 2), l == 0 ? 1 : 0);
  auto for_rect = [&](const int* a, const int* b, auto&& fn) {
    int p[3];
    for (p[2] = a[2]; p[2] < b[2]; p[2]++)
      for (p[1] = a[1]; p[1] < b[1]; p[1]++)
        for (p[0] = a[0]; p[0] < b[0]; p[0]++) fn(p);
  };
  for (int k = 0; k < nb; k++) {  // the region of the next level
    const int l = box_level[k];
    int a[3] = {0, 0, 0}, b[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) a[d] = 3 * lo[3 * k + d], b[d] = 3 * hi[3 * k + d];
    if (a[0] >= b[0] || a[1] >= b[1] || a[2] >= b[2]) return "empty box";
    for_rect(a, b, [&](const int* p) { st[l + 1][idx(l + 1, p)] = 1; });
  }
  const char* err = nullptr;
  for (int k = 0; k < nb && !err; k++) {  // margins, then mark refined
    const int l = box_level[k];
    int a[3] = {0, 0, 0}, b[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) a[d] = lo[3 * k + d] - 1, b[d] = hi[3 * k + d] + 1;
    for_rect(a, b, [&](const int* p) {
      if (!inrect(l, p) || st[l][idx(l, p)] == 0) err = "each box must lie inside its level's region with one cell around it";
    });
  }
  if (err) return err;
  for (int k = 0; k < nb; k++) {
    const int l = box_level[k];
    int a[3] = {0, 0, 0}, b[3] = {1, 1, 1};
    for (int d = 0; d < dim; d++) a[d] = lo[3 * k + d], b[d] = hi[3 * k + d];
    for_rect(a, b, [&](const int* p) { st[l][idx(l, p)] = 2; });
  }
  auto state = [&](int l, const int* p) { return inrect(l, p) ? st[l][idx(l, p)] : (unsigned char)0; };
  // slots: cells level by level (x fastest), then ancestors, then descendants
  std::vector<std::vector<int>> slot(L);
  int n = 0;
  for (int l = 0; l < L; l++) {
    slot[l].assign(st[l].size(), -1);
    for_rect(r0[l].data(), r1[l].data(), [&](const int* p) {
      if (st[l][idx(l, p)] == 1) {
        slot[l][idx(l, p)] = n++;
        t.level.push_back(l);
        t.pos.insert(t.pos.end(), {p[0], p[1], p[2]});
      }
    });
  }
  t.ncells = n;
  t.anc0 = n;
  auto nb_pos = [&](int l, const int* p, int d, int s, int* q) {  // the neighbour across face 2d+s
    q[0] = p[0], q[1] = p[1], q[2] = p[2];
    q[d] += s ? 1 : -1;
    if (l == 0 && bc[2 * d] == EXA_BC_PERIODIC) q[d] = (q[d] + cells[d]) % cells[d];
  };
  for (int l = 0; l + 1 < L; l++)  // ancestors: refined positions facing a cell
    for_rect(r0[l].data(), r1[l].data(), [&](const int* p) {
      if (st[l][idx(l, p)] != 2) return;
      bool faces_cell = false;
      for (int d = 0; d < dim; d++)
        for (int s = 0; s < 2; s++) {
          int q[3];
          nb_pos(l, p, d, s, q);
          faces_cell |= state(l, q) == 1;
        }
      if (faces_cell) slot[l][idx(l, p)] = n++, t.nanc++;
    });
  for (int l = 0; l < L; l++)
    for_rect(r0[l].data(), r1[l].data(), [&](const int* p) {
      const unsigned char sp = st[l][idx(l, p)];
      if (sp == 0) return;
      const int me = slot[l][idx(l, p)];  // -1: refined and facing no cell
      for (int d = 0; d < dim; d++) {
        int q[3];
        nb_pos(l, p, d, 1, q);
        const unsigned char sq = state(l, q);
        if (sq != 0 && !(sp == 2 && sq == 2)) {  // same-level pair with at least one cell
          t.fl.push_back(me);
          t.fr.push_back(slot[l][idx(l, q)]);
          t.fd.push_back(d);
        }
        if (sp != 1) continue;
        for (int s = 0; s < 2; s++) {
          int r[3];
          nb_pos(l, p, d, s, r);
          if (state(l, r) != 0) continue;
          if (l == 0) {  // a domain face
            t.bcell.push_back(me);
            t.bface.push_back(2 * d + s);
            t.bkind.push_back(bc[2 * d + s]);
            continue;
          }
          // a cell on its region's face: a descendant across it (the coarse
          // neighbour's virtual child), with the face transfers
          int sub[2] = {0, 0}, ns = 0;
          for (int e = 0; e < dim; e++)
            if (e != d) sub[ns++] = p[e] % 3;
          const int parent[3] = {p[0] / 3, p[1] / 3, dim == 3 ? p[2] / 3 : 0};
          const int rparent[3] = {r[0] / 3, r[1] / 3, dim == 3 ? r[2] / 3 : 0};
          const int face = 2 * d + s, dface = 2 * d + (1 - s), desc = n++;
          t.fl.push_back(s == 0 ? desc : me);
          t.fr.push_back(s == 0 ? me : desc);
          t.fd.push_back(d);
          t.rf.push_back(me * D2 + face);
          t.rc.push_back(slot[l - 1][idx(l - 1, parent)] * D2 + face);
          t.ridx.push_back(sub[0]);
          t.ridx.push_back(sub[1]);
          t.pf.push_back(desc * D2 + dface);
          t.pc.push_back(slot[l - 1][idx(l - 1, rparent)] * D2 + dface);
          t.pidx.push_back(sub[0]);
          t.pidx.push_back(sub[1]);
        }
      }
    });
  t.nslots = n;
  t.maps.resize(L);
  for (int l = 0; l < L; l++) {
    LevelMap& mp = t.maps[l];
    mp.r0 = r0[l];
    mp.r1 = r1[l];
    mp.st = st[l];
    mp.cell.assign(st[l].size(), -1);
    for (size_t i = 0; i < st[l].size(); i++)
      if (st[l][i] == 1) mp.cell[i] = slot[l][i];
  }
  return nullptr;
}
}  // namespace

int exa_mesh_create_boxes(const exa_solver* s, const int* cells, const double* offset, const double* size,
                          const int* bc, int nboxes, const int* box_level, const int* box_lo, const int* box_hi,
                          exa_mesh** out) {
  if (!s || !cells || !offset || !size || !out || (nboxes > 0 && (!box_level || !box_lo || !box_hi)))
    return fail(EXA_ERR_ARG, "exa_mesh_create_boxes: null argument");
  if (nboxes < 0 || nboxes > 4096) return fail(EXA_ERR_ARG, "exa_mesh_create_boxes: 0 to 4096 refined boxes");
  const int dim = s->k.dim, D2 = 2 * dim;
  std::unique_ptr<exa_mesh> m(new exa_mesh());
  m->s = s;
  m->dim = dim;
  for (int d = 0; d < dim; d++) {
    if (cells[d] < 3 || !(size[d] > 0)) return fail(EXA_ERR_ARG, "exa_mesh_create_boxes: bad grid");
    m->cells[d] = cells[d];
    m->offset[d] = offset[d];
    m->size[d] = size[d];
    m->geo.dx[d] = size[d] / cells[d];
  }
  for (int d = dim; d < 3; d++) m->geo.dx[d] = 1.0;
  for (int f = 0; f < 6; f++) {
    const int k = bc && f < 2 * dim ? bc[f] : EXA_BC_PERIODIC;
    if (k != EXA_BC_PERIODIC && k != EXA_BC_OUTFLOW && k != EXA_BC_REFLECTIVE)
      return fail(EXA_ERR_ARG, "exa_mesh_create_boxes: unknown boundary kind");
    if (f % 2 == 1 && (k == EXA_BC_PERIODIC) != (m->bc[f - 1] == EXA_BC_PERIODIC))
      return fail(EXA_ERR_ARG, "exa_mesh_create_boxes: periodic must be set on both faces of an axis");
    m->bc[f] = k;
  }
  NestedTopo t;
  if (const char* err = boxes_topology(dim, cells, m->bc, nboxes, box_level, box_lo, box_hi, t))
    return fail(EXA_ERR_ARG, std::string("exa_mesh_create_boxes: ") + err);
  {  // domain faces grouped by kind: outflow, then reflective
    std::vector<int> bc2, bf2;
    for (int kd = 0; kd < 2; kd++) {
      m->boff[kd] = (int)bc2.size();
      for (size_t i = 0; i < t.bcell.size(); i++)
        if (t.bkind[i] == kd) bc2.push_back(t.bcell[i]), bf2.push_back(t.bface[i]);
      m->nbfaces[kd] = (int)bc2.size() - m->boff[kd];
    }
    t.bcell.swap(bc2);
    t.bface.swap(bf2);
  }
  const int L = t.L;
  m->ncells = t.ncells;
  m->nfaces = (int)t.fl.size();
  m->ref.on = true;
  m->ref.nlev = L;
  m->ref.anc0 = t.anc0;
  m->ref.nanc = t.nanc;
  m->ref.nres = (int)t.rf.size();
  m->ref.npro = (int)t.pf.size();
  // each level's width is its parent level's divided by 3 (as a spacetree
  // computes the width of a child cell)
  std::vector<double> ldx(3 * (size_t)L);
  for (int d = 0; d < 3; d++) ldx[d] = m->geo.dx[d];
  for (int l = 1; l < L; l++)
    for (int d = 0; d < 3; d++) ldx[3 * l + d] = d < dim ? ldx[3 * (l - 1) + d] / 3.0 : 1.0;
  std::vector<int> ones(std::max<size_t>(1, t.rf.size() + t.pf.size()), 1);
  const size_t P = s->k.P, F = s->k.F, nV = s->k.nvar, nD = s->k.nvar + s->k.npar;
  const size_t n = m->ncells, ns = t.nslots;
  EXA_CUDA(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking));
  cudaStream_t st = m->stream;
  auto ia = [&](int** p, size_t cnt) { return salloc(p, std::max<size_t>(1, cnt) * 4, st); };
  bool ok = salloc(&m->luh, n * P * nD * 8, st) && salloc(&m->lduh, n * P * nV * 8, st) &&
            salloc(&m->lQhbnd, ns * D2 * F * nD * 8, st) && salloc(&m->lFhbnd, ns * D2 * F * nV * 8, st) &&
            salloc(&m->scal, 8 * 8, st) && ia(&m->iters, n) && ia(&m->fl, t.fl.size()) && ia(&m->fr, t.fl.size()) &&
            ia(&m->fd, t.fl.size()) && ia(&m->bcell, t.bcell.size()) && ia(&m->bface, t.bcell.size()) &&
            salloc(&m->sweeps, 8, st) && salloc(&m->ref.lv, 3 * (size_t)L * 8, st) && ia(&m->ref.inst, n) &&
            salloc(&m->ref.inst_dx, ldx.size() * 8, st) && ia(&m->ref.res_f, t.rf.size()) &&
            ia(&m->ref.res_c, t.rf.size()) && ia(&m->ref.res_ld, t.rf.size()) && ia(&m->ref.res_idx, t.ridx.size()) &&
            ia(&m->ref.pro_f, t.pf.size()) && ia(&m->ref.pro_c, t.pf.size()) && ia(&m->ref.pro_ld, t.pf.size()) &&
            ia(&m->ref.pro_idx, t.pidx.size());
  if (!ok) {
    cudaGetLastError();
    mesh_free(m.get());
    return fail(EXA_ERR_NOMEM, "exa_mesh_create_boxes: device allocation failed");
  }
  auto up = [&](void* dst, const void* src, size_t bytes) {
    return bytes == 0 || cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess;
  };
  ok = up(m->fl, t.fl.data(), t.fl.size() * 4) && up(m->fr, t.fr.data(), t.fr.size() * 4) &&
       up(m->fd, t.fd.data(), t.fd.size() * 4) && up(m->ref.inst, t.level.data(), n * 4) &&
       up(m->ref.inst_dx, ldx.data(), ldx.size() * 8) && up(m->ref.res_f, t.rf.data(), t.rf.size() * 4) &&
       up(m->ref.res_c, t.rc.data(), t.rc.size() * 4) && up(m->ref.res_ld, ones.data(), t.rf.size() * 4) &&
       up(m->ref.res_idx, t.ridx.data(), t.ridx.size() * 4) && up(m->ref.pro_f, t.pf.data(), t.pf.size() * 4) &&
       up(m->ref.pro_c, t.pc.data(), t.pc.size() * 4) && up(m->ref.pro_ld, ones.data(), t.pf.size() * 4) &&
       up(m->ref.pro_idx, t.pidx.data(), t.pidx.size() * 4) && up(m->bcell, t.bcell.data(), t.bcell.size() * 4) &&
       up(m->bface, t.bface.data(), t.bface.size() * 4);
  if (!ok) {
    cudaStreamSynchronize(st);
    mesh_free(m.get());
    return fail(EXA_ERR_CUDA, "exa_mesh_create_boxes: upload failed");
  }

  m->geo.inst = m->ref.inst;
  m->geo.inst_dx = m->ref.inst_dx;
  m->ref.level = t.level;
  m->ref.pos = t.pos;
  m->ref.ldx = ldx;
  m->ref.maps = std::move(t.maps);
  EXA_CUDA(cudaMemsetAsync(m->luh, 0, n * P * nD * 8, st));
  EXA_CUDA(cudaMemsetAsync(m->lduh, 0, n * P * nV * 8, st));
  EXA_CUDA(cudaMemsetAsync(m->lQhbnd, 0, ns * D2 * F * nD * 8, st));
  EXA_CUDA(cudaMemsetAsync(m->lFhbnd, 0, ns * D2 * F * nV * 8, st));
  EXA_CUDA(cudaMemsetAsync(m->sweeps, 0, 8, st));
  EXA_CUDA(cudaStreamSynchronize(st));  // the host vectors go out of scope
  if (int rc = mesh_centres(m.get(), m->ref.pos, &m->ref.level, m->ref.ldx)) {
    mesh_free(m.get());
    return rc;
  }
  *out = m.release();
  return EXA_OK;
}

int exa_mesh_create_nested(const exa_solver* s, const int* cells, const double* offset, const double* size,
                           const int* bc, int nboxes, const int* box_lo, const int* box_hi, exa_mesh** out) {
  if (nboxes < 1 || nboxes > 8) return fail(EXA_ERR_ARG, "exa_mesh_create_nested: 1 to 8 refined boxes");
  const int level[8] = {0, 1, 2, 3, 4, 5, 6, 7};
  return exa_mesh_create_boxes(s, cells, offset, size, bc, nboxes, level, box_lo, box_hi, out);
}

int exa_mesh_create_refined(const exa_solver* s, const int* cells, const double* offset, const double* size,
                            const int* box_lo, const int* box_hi, exa_mesh** out) {
  return exa_mesh_create_nested(s, cells, offset, size, nullptr, 1, box_lo, box_hi, out);
}

int exa_mesh_destroy(exa_mesh* m) {
  if (!m) return EXA_OK;
  mesh_free(m);
  delete m;
  return EXA_OK;
}

int exa_mesh_num_cells(const exa_mesh* m, int* n) {
  if (!m || !n) return fail(EXA_ERR_ARG, "exa_mesh_num_cells: null argument");
  *n = m->ncells;
  return EXA_OK;
}

int exa_mesh_set_solution(exa_mesh* m, const double* h) {
  if (!m || !h) return fail(EXA_ERR_ARG, "exa_mesh_set_solution: null argument");
  const size_t bytes = (size_t)m->ncells * m->s->k.P * (m->s->k.nvar + m->s->k.npar) * 8;
  EXA_CUDA(cudaMemcpyAsync(m->luh, h, bytes, cudaMemcpyHostToDevice, m->stream));
  EXA_CUDA(cudaStreamSynchronize(m->stream));
  return EXA_OK;
}

int exa_mesh_get_solution(exa_mesh* m, double* h) {
  if (!m || !h) return fail(EXA_ERR_ARG, "exa_mesh_get_solution: null argument");
  const size_t bytes = (size_t)m->ncells * m->s->k.P * (m->s->k.nvar + m->s->k.npar) * 8;
  EXA_CUDA(cudaMemcpyAsync(h, m->luh, bytes, cudaMemcpyDeviceToHost, m->stream));
  EXA_CUDA(cudaStreamSynchronize(m->stream));
  return EXA_OK;
}

int exa_mesh_copy_solution(exa_mesh* m, void* host, size_t nbytes, int to_device) {
  if (!m || !host) return fail(EXA_ERR_ARG, "exa_mesh_copy_solution: null argument");
  const size_t bytes = (size_t)m->ncells * m->s->k.P * (m->s->k.nvar + m->s->k.npar) * 8;
  if (nbytes != bytes) return fail(EXA_ERR_ARG, "exa_mesh_copy_solution: nbytes does not match the solution size");
  if (to_device)
    EXA_CUDA(cudaMemcpyAsync(m->luh, host, bytes, cudaMemcpyHostToDevice, m->stream));
  else
    EXA_CUDA(cudaMemcpyAsync(host, m->luh, bytes, cudaMemcpyDeviceToHost, m->stream));
  return EXA_OK;
}

// The predictor of every cell; fused time stepping runs it with its own step
// size (scal[5]) and, for the rerun, only when *count (device) is not 0.
// The step size the kernels read and the new step's min-reduction target
// (per level on a refined mesh).
static double* mesh_dt(exa_mesh* m) { return m->ref.on ? m->ref.lv : m->scal + 0; }
static double* mesh_dt_min(exa_mesh* m) { return m->ref.on ? m->ref.lv + m->ref.nlev : m->scal + 1; }

// Refined mesh, after every predictor: the ancestors' faces are zeroed and
// receive the restriction of their fine children's extrapolated states and
// fluxes (restrictToTopMostParent, ADERDGSolver.cpp:2465-2515, after
// prepareFaceDataOfAncestor :2300-2331); the descendants' faces receive the
// prolongation of their coarse parent's (prolongateFaceDataToDescendant
// :2334-2382). The Riemann solves then pair fine cells with descendants and
// coarse cells with ancestors (solveRiemannProblemAtInterface :2789, any
// pair with at least one cell).
static int mesh_amr_faces(exa_mesh* m) {
  const KernelSet& k = m->s->k;
  const size_t D2 = 2 * m->dim, nD = k.nvar + k.npar;
  EXA_CUDA(cudaMemsetAsync(m->lQhbnd + (size_t)m->ref.anc0 * D2 * k.F * nD, 0, (size_t)m->ref.nanc * D2 * k.F * nD * 8,
                           m->stream));
  EXA_CUDA(cudaMemsetAsync(m->lFhbnd + (size_t)m->ref.anc0 * D2 * k.F * k.nvar, 0,
                           (size_t)m->ref.nanc * D2 * k.F * k.nvar * 8, m->stream));
  int rc = k.amr_face(m->lQhbnd, m->lFhbnd, m->lQhbnd, m->lFhbnd, m->ref.nres, m->ref.res_f, m->ref.res_c,
                      m->ref.res_ld, m->ref.res_idx, 1, m->stream);
  if (rc) return rc;
  return k.amr_face(m->lQhbnd, m->lFhbnd, m->lQhbnd, m->lFhbnd, m->ref.npro, m->ref.pro_f, m->ref.pro_c,
                    m->ref.pro_ld, m->ref.pro_idx, 0, m->stream);
}

// after_update: the fused scheme's predictor right after the update, whose
// solution carries the predictor time stamp scal[4]; every other predictor
// call starts from the corrector time stamp scal[2] (point sources)
static int mesh_predict(exa_mesh* m, const int* count = nullptr, bool after_update = false) {
  const KernelSet& k = m->s->k;
  PhaseTimer pt(m, 0);
  m->phase_launches[0] += 2;
  double* dt = m->fused ? (m->ref.on ? m->ref.lv + 2 * m->ref.nlev : m->scal + 5) : mesh_dt(m);
  Geometry g = m->geo;
  if (k.point_source) {
    g.time = m->scal + (after_update ? 4 : 2);
    for (int i = 0; i < 6; i++) g.ps[i] = m->s->ps[i];
  }
  int rc = k.predictor(m->luh, m->lQhbnd, m->lFhbnd, m->lduh, m->iters, dt, g,
                       m->ncells, nullptr, count, PredictorTemps{}, false, m->sweeps, m->s->variant, m->stream);
  if (rc || !m->ref.on) return rc;
  m->phase_launches[0] += 3;
  return mesh_amr_faces(m);
}

// Fused time stepping scalars: [0] corrector step, [1] min-reduction target,
// [2] corrector time stamp, [3] steps, [4] predictor time stamp, [5]
// predictor step, [6] predictor reruns (ADERDGSolver's _minCorrector*/
// _minPredictor*). Arithmetic in round-to-nearest operations, as the
// reference's unfused evaluation.
// Refined meshes (lv != NULL, L levels): the min-reduction targets are
// lv[L..2L-1], and the levels' corrector and predictor steps lv[0..L-1] and
// lv[2L..3L-1] are copies of scal[0] and scal[5].
__device__ double fused_take_min(double* scal, double* lv, int L) {
  const double big = __longlong_as_double(0x7fefffffffffffffll);
  if (!lv) {
    const double s = scal[1];
    scal[1] = big;
    return s;
  }
  double s = big;
  for (int l = 0; l < L; l++) {
    s = (lv[L + l] < s) ? lv[L + l] : s;
    lv[L + l] = big;
  }
  return s;
}
__device__ void fused_copy_levels(const double* scal, double* lv, int L) {
  if (!lv) return;
  for (int l = 0; l < L; l++) {
    lv[l] = scal[0];
    lv[2 * L + l] = scal[5];
  }
}

__global__ void fused_init_kernel(double* scal, double* lv, int L) {
  const double s0 = fused_take_min(scal, lv, L);  // min admissible step of the initial data
  scal[0] = s0;
  scal[5] = s0;
  scal[4] = __dadd_rn(scal[2], s0);
  scal[6] = 0.0;
  fused_copy_levels(scal, lv, L);
}

// end of a fused step (SolutionUpdate::endIteration,
// TimeStepSizeComputation::reinitialiseTimeStepDataIfLastPredictorTimeStepSizeWasInstable,
// ADERDGSolver::startNewTimeStep; TimeStepSizeComputation.cpp:167-204,
// ADERDGSolver.cpp:559-592): s = min stable step after the update; a
// predictor step above s is replaced by w s (and the predictor rerun), else
// the next estimate is the mean of the used step and w s
__global__ void fused_advance_kernel(double* scal, double w, int* rerun, int ncells, double* lv, int L) {
  const double s = fused_take_min(scal, lv, L);
  double next = __longlong_as_double(0x7fefffffffffffffll);
  next = (s < next) ? s : next;
  double pdt = scal[5];
  const double used = (pdt == 0.0) ? s : pdt;
  const bool unstable = used > s;
  if (unstable) {
    const double ws = __dmul_rn(w, s);
    next = (ws < next) ? ws : next;
    pdt = ws;
  } else {
    const double avg = __dmul_rn(0.5, __dadd_rn(used, __dmul_rn(w, s)));
    next = (avg < next) ? avg : next;
  }
  scal[2] = scal[4];
  scal[0] = pdt;
  scal[4] = __dadd_rn(scal[4], pdt);
  scal[5] = next;
  scal[3] += 1.0;
  if (unstable) scal[6] += 1.0;
  *rerun = unstable ? ncells : 0;
  fused_copy_levels(scal, lv, L);
}

int exa_mesh_init_fused(exa_mesh* m, double t0, double weight) {
  if (!m || !(weight > 0.0) || weight > 1.0) return fail(EXA_ERR_ARG, "exa_mesh_init_fused: bad argument");
  const KernelSet& k = m->s->k;
  if (!m->rerun && !salloc(&m->rerun, sizeof(int), m->stream)) {
    cudaGetLastError();
    m->rerun = nullptr;
    return fail(EXA_ERR_NOMEM, "exa_mesh_init_fused: device allocation failed");
  }
  m->fused = true;
  m->weight = weight;
  init_scalars_kernel<<<1, 1, 0, m->stream>>>(m->scal, t0);
  EXA_LAUNCHED();
  if (m->ref.on) {
    level_reset_kernel<<<1, 1, 0, m->stream>>>(m->ref.lv, m->ref.nlev);
    EXA_LAUNCHED();
  }
  EXA_CUDA(cudaMemsetAsync(m->sweeps, 0, 8, m->stream));
  EXA_CUDA(cudaMemsetAsync(m->rerun, 0, sizeof(int), m->stream));
  int rc = k.corrector(m->luh, nullptr, nullptr, nullptr, mesh_dt_min(m), m->geo, m->ncells, nullptr, 0, nullptr,
                       m->stream);
  if (rc) return rc;
  fused_init_kernel<<<1, 1, 0, m->stream>>>(m->scal, m->ref.on ? m->ref.lv : nullptr, m->ref.nlev);
  EXA_LAUNCHED();
  rc = mesh_predict(m);
  if (rc) return rc;
  m->initialised = true;
  return EXA_OK;
}

int exa_mesh_fused_state(exa_mesh* m, double* predictor_dt, long long* reruns) {
  if (!m) return fail(EXA_ERR_ARG, "exa_mesh_fused_state: null mesh");
  if (!m->fused) return fail(EXA_ERR_STATE, "exa_mesh_fused_state: the mesh is not in fused time stepping");
  double h[7];
  EXA_CUDA(cudaMemcpyAsync(h, m->scal, sizeof(h), cudaMemcpyDeviceToHost, m->stream));
  EXA_CUDA(cudaStreamSynchronize(m->stream));
  if (predictor_dt) *predictor_dt = h[5];
  if (reruns) *reruns = (long long)h[6];
  return EXA_OK;
}

int exa_mesh_init(exa_mesh* m, double t0) {
  if (!m) return fail(EXA_ERR_ARG, "exa_mesh_init: null mesh");
  const KernelSet& k = m->s->k;
  m->fused = false;
  init_scalars_kernel<<<1, 1, 0, m->stream>>>(m->scal, t0);
  EXA_LAUNCHED();
  if (m->ref.on) {
    level_reset_kernel<<<1, 1, 0, m->stream>>>(m->ref.lv, m->ref.nlev);
    EXA_LAUNCHED();
  }
  EXA_CUDA(cudaMemsetAsync(m->sweeps, 0, 8, m->stream));
  // first admissible step from the initial data, then the first predictor
  int rc = k.corrector(m->luh, nullptr, nullptr, nullptr, mesh_dt_min(m), m->geo, m->ncells, nullptr, 0, nullptr,
                       m->stream);
  if (rc) return rc;
  if (m->ref.on)
    level_take_kernel<<<1, 1, 0, m->stream>>>(m->scal, m->ref.lv, m->ref.nlev);
  else
    take_dt_kernel<<<1, 1, 0, m->stream>>>(m->scal);
  EXA_LAUNCHED();
  rc = mesh_predict(m);
  if (rc) return rc;
  m->initialised = true;
  return EXA_OK;
}

static int mesh_one_step(exa_mesh* m) {
  const KernelSet& k = m->s->k;
  int rc;
  {
    PhaseTimer pt(m, 1);
    rc = k.riemann(m->lQhbnd, m->lFhbnd, m->fl, m->fr, m->fd, m->nfaces, nullptr, m->stream);
    if (rc) return rc;
    m->phase_launches[1] += m->nfaces > 0;
    for (int kd = 0; kd < 2; kd++) {
      rc = k.boundary(m->lQhbnd, m->lFhbnd, m->bcell + m->boff[kd], m->bface + m->boff[kd], m->nbfaces[kd], kd,
                      nullptr, m->stream);
      if (rc) return rc;
      m->phase_launches[1] += m->nbfaces[kd] > 0;
    }
  }
  {
    PhaseTimer pt(m, 2);
    rc = k.corrector(m->luh, m->lduh, m->lFhbnd, mesh_dt(m), mesh_dt_min(m), m->geo, m->ncells, nullptr, 1, nullptr,
                     m->stream);
    if (rc) return rc;
    m->phase_launches[2] += 1;
  }
  if (m->fused) {
    // fused time stepping: the predictor of the next step runs with its own
    // step size right after the update (no global reduction in between),
    // then the step bookkeeping, then the rerun, which does nothing unless
    // needed (its blocks return at once when the device count is 0)
    rc = mesh_predict(m, nullptr, true);
    if (rc) return rc;
    {
      PhaseTimer pt(m, 3);
      fused_advance_kernel<<<1, 1, 0, m->stream>>>(m->scal, m->weight, m->rerun, m->ncells,
                                                   m->ref.on ? m->ref.lv : nullptr, m->ref.nlev);
      EXA_LAUNCHED();
      m->phase_launches[3] += 1;
    }
    return mesh_predict(m, m->rerun);
  }
  {
    PhaseTimer pt(m, 3);
    if (m->ref.on)
      level_advance_kernel<<<1, 1, 0, m->stream>>>(m->scal, m->ref.lv, m->ref.nlev);
    else
      advance_kernel<<<1, 1, 0, m->stream>>>(m->scal);
    EXA_LAUNCHED();
    m->phase_launches[3] += 1;
  }
  return mesh_predict(m);
}

int exa_mesh_step(exa_mesh* m, int nsteps) {
  if (!m) return fail(EXA_ERR_ARG, "exa_mesh_step: null mesh");
  if (!m->initialised) return fail(EXA_ERR_STATE, "exa_mesh_step: call exa_mesh_init first");
  for (int i = 0; i < nsteps; i++) {
    int rc = mesh_one_step(m);
    if (rc) return rc;
  }
  return EXA_OK;
}

int exa_mesh_step_io(exa_mesh* m, const void* host_in, int nin, void* host_out, int nout, size_t nbytes,
                     int nsteps) {
  if (!m || !host_in || !host_out || nin < 1 || nout < 1 || nsteps < 0)
    return fail(EXA_ERR_ARG, "exa_mesh_step_io: bad argument");
  if (!m->initialised) return fail(EXA_ERR_STATE, "exa_mesh_step_io: call exa_mesh_init first");
  const size_t bytes = (size_t)m->ncells * m->s->k.P * (m->s->k.nvar + m->s->k.npar) * 8;
  if (nbytes != bytes) return fail(EXA_ERR_ARG, "exa_mesh_step_io: nbytes does not match the solution size");
  if (!m->io_in) {
    EXA_CUDA(cudaStreamCreateWithFlags(&m->io_in, cudaStreamNonBlocking));
    EXA_CUDA(cudaStreamCreateWithFlags(&m->io_out, cudaStreamNonBlocking));
    for (cudaEvent_t* e : {&m->in_ready, &m->in_free, &m->out_ready, &m->out_free})
      EXA_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    if (!salloc(&m->stage_in, bytes, m->stream) || !salloc(&m->stage_out, bytes, m->stream)) {
      cudaGetLastError();
      return fail(EXA_ERR_NOMEM, "exa_mesh_step_io: device allocation failed");
    }
    // the staging buffers exist before either copy stream touches them
    EXA_CUDA(cudaEventRecord(m->in_free, m->stream));
    EXA_CUDA(cudaEventRecord(m->out_free, m->stream));
  }
  const char* in = static_cast<const char*>(host_in);
  char* out = static_cast<char*>(host_out);
  for (int k = 0; k < nsteps; k++) {
    // input k: once the previous input has left the staging buffer
    EXA_CUDA(cudaStreamWaitEvent(m->io_in, m->in_free, 0));
    EXA_CUDA(cudaMemcpyAsync(m->stage_in, in + (size_t)(k % nin) * bytes, bytes, cudaMemcpyHostToDevice, m->io_in));
    EXA_CUDA(cudaEventRecord(m->in_ready, m->io_in));
    EXA_CUDA(cudaStreamWaitEvent(m->stream, m->in_ready, 0));
    EXA_CUDA(cudaMemcpyAsync(m->luh, m->stage_in, bytes, cudaMemcpyDeviceToDevice, m->stream));
    EXA_CUDA(cudaEventRecord(m->in_free, m->stream));
    int rc = mesh_one_step(m);
    if (rc) return rc;
    // result k: once the previous result has left the staging buffer
    EXA_CUDA(cudaStreamWaitEvent(m->stream, m->out_free, 0));
    EXA_CUDA(cudaMemcpyAsync(m->stage_out, m->luh, bytes, cudaMemcpyDeviceToDevice, m->stream));
    EXA_CUDA(cudaEventRecord(m->out_ready, m->stream));
    EXA_CUDA(cudaStreamWaitEvent(m->io_out, m->out_ready, 0));
    EXA_CUDA(cudaMemcpyAsync(out + (size_t)(k % nout) * bytes, m->stage_out, bytes, cudaMemcpyDeviceToHost,
                             m->io_out));
    EXA_CUDA(cudaEventRecord(m->out_free, m->io_out));
  }
  // the mesh stream (what exa_mesh_synchronize and the caller's events see)
  // completes after the last result is on the host
  EXA_CUDA(cudaStreamWaitEvent(m->stream, m->out_free, 0));
  return EXA_OK;
}

int exa_mesh_state(exa_mesh* m, double* t, double* dt, long long* steps, long long* sweeps) {
  if (!m) return fail(EXA_ERR_ARG, "exa_mesh_state: null mesh");
  double h[4];
  unsigned long long sw = 0;
  EXA_CUDA(cudaMemcpyAsync(h, m->scal, sizeof(h), cudaMemcpyDeviceToHost, m->stream));
  EXA_CUDA(cudaMemcpyAsync(&sw, m->sweeps, 8, cudaMemcpyDeviceToHost, m->stream));
  EXA_CUDA(cudaStreamSynchronize(m->stream));
  if (t) *t = h[2];
  if (dt) *dt = h[0];
  if (steps) *steps = (long long)h[3];
  if (sweeps) *sweeps = (long long)sw;
  return EXA_OK;
}

int exa_mesh_validate(exa_mesh* m, long long* nonfinite_cells) {
  if (!m || !nonfinite_cells) return fail(EXA_ERR_ARG, "exa_mesh_validate: null argument");
  const KernelSet& k = m->s->k;
  const size_t n = m->ncells, P = k.P, F = k.F, nV = k.nvar, nD = k.nvar + k.npar, D2 = 2 * m->dim;
  int* flag = nullptr;
  unsigned long long* cnt = nullptr;
  if (!salloc(&flag, n * 4, m->stream) || !salloc(&cnt, 8, m->stream)) {
    cudaGetLastError();
    if (flag) sfree(flag, m->stream);
    return fail(EXA_ERR_NOMEM, "exa_mesh_validate: device allocation failed");
  }
  EXA_CUDA(cudaMemsetAsync(flag, 0, n * 4, m->stream));
  EXA_CUDA(cudaMemsetAsync(cnt, 0, 8, m->stream));
  const struct {
    const double* a;
    size_t per;
  } arrays[4] = {{m->luh, P * nD}, {m->lduh, P * nV}, {m->lQhbnd, D2 * F * nD}, {m->lFhbnd, D2 * F * nV}};
  for (const auto& x : arrays) {
    const size_t total = n * x.per;
    const int grid = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    if (total) nonfinite_flag_kernel<<<grid, 256, 0, m->stream>>>(x.a, x.per, total, flag);
    EXA_LAUNCHED();
  }
  count_flags_kernel<<<std::max(1, std::min((int)((n + 255) / 256), 148 * 4)), 256, 0, m->stream>>>(flag, (int)n, cnt);
  EXA_LAUNCHED();
  unsigned long long h = 0;
  EXA_CUDA(cudaMemcpyAsync(&h, cnt, 8, cudaMemcpyDeviceToHost, m->stream));
  sfree(flag, m->stream);
  sfree(cnt, m->stream);
  EXA_CUDA(cudaStreamSynchronize(m->stream));
  *nonfinite_cells = (long long)h;
  return EXA_OK;
}

// Data of a regridded mesh (ADERDGSolver::prolongateVolumeData /
// restrictVolumeData, exahype/solvers/ADERDGSolver.cpp:1437-1470,1694-1735,
// volumeUnknownsProlongation / volumeUnknownsRestriction): a new cell that
// was a cell keeps its data; one inside a coarser old cell gets that cell's
// prolongation (levelDelta = the level difference); one covering finer old
// cells gets the sum of their restrictions. Then the time stamp and step
// count are kept, the admissible step is recomputed from the new solution
// and the predictor runs on every cell.
int exa_mesh_regrid(exa_mesh* m, int nboxes, const int* box_level, const int* box_lo, const int* box_hi) {
  if (!m) return fail(EXA_ERR_ARG, "exa_mesh_regrid: null mesh");
  if (!m->ref.on) return fail(EXA_ERR_UNSUPPORTED, "exa_mesh_regrid: create the mesh with exa_mesh_create_boxes");
  if (!m->initialised) return fail(EXA_ERR_STATE, "exa_mesh_regrid: call exa_mesh_init first");
  if (m->fused) return fail(EXA_ERR_UNSUPPORTED, "exa_mesh_regrid: meshes in fused time stepping are not regridded");
  exa_mesh* nm = nullptr;
  int rc = exa_mesh_create_boxes(m->s, m->cells, m->offset, m->size, m->bc, nboxes, box_level, box_lo, box_hi, &nm);
  if (rc) return rc;
  std::unique_ptr<exa_mesh, int (*)(exa_mesh*)> guard(nm, exa_mesh_destroy);
  const KernelSet& k = m->s->k;
  const int dim = m->dim, oldL = (int)m->ref.maps.size();
  std::vector<int> cto, cfrom, pf, pc, pld, pidx, rfine, rcoarse, rld, ridx;
  for (int c = 0; c < nm->ncells; c++) {
    const int l = nm->ref.level[c];
    const int* p = &nm->ref.pos[3 * (size_t)c];
    int lv = std::min(l, oldL - 1), a[3] = {p[0], p[1], p[2]};
    for (int i = lv; i < l; i++)
      for (int d = 0; d < dim; d++) a[d] /= 3;
    // the finest old level whose region holds this position's ancestor
    while (lv > 0 && !(m->ref.maps[lv].inside(a) && m->ref.maps[lv].st[m->ref.maps[lv].at(a)] != 0)) {
      lv--;
      for (int d = 0; d < dim; d++) a[d] /= 3;
    }
    const LevelMap& om = m->ref.maps[lv];
    const unsigned char sa = om.st[om.at(a)];
    if (sa == 1 && lv == l) {  // the same cell
      cto.push_back(c);
      cfrom.push_back(om.cell[om.at(a)]);
    } else if (sa == 1) {  // inside a coarser old cell
      const int ld = l - lv;
      int f = 1;
      for (int i = 0; i < ld; i++) f *= 3;
      pf.push_back(c);
      pc.push_back(om.cell[om.at(a)]);
      pld.push_back(ld);
      for (int d = 0; d < 3; d++) pidx.push_back(d < dim ? p[d] - a[d] * f : 0);
    } else {  // refined in the old mesh: the finer old cells inside it
      for (int l2 = l + 1; l2 < oldL; l2++) {
        const LevelMap& fm = m->ref.maps[l2];
        int f = 1;
        for (int i = l; i < l2; i++) f *= 3;
        int q0[3] = {0, 0, 0}, q1[3] = {1, 1, 1};
        for (int d = 0; d < dim; d++) q0[d] = std::max(p[d] * f, fm.r0[d]), q1[d] = std::min((p[d] + 1) * f, fm.r1[d]);
        int q[3];
        for (q[2] = q0[2]; q[2] < q1[2]; q[2]++)
          for (q[1] = q0[1]; q[1] < q1[1]; q[1]++)
            for (q[0] = q0[0]; q[0] < q1[0]; q[0]++) {
              if (fm.st[fm.at(q)] != 1) continue;
              rfine.push_back(fm.cell[fm.at(q)]);
              rcoarse.push_back(c);
              rld.push_back(l2 - l);
              for (int d = 0; d < 3; d++) ridx.push_back(d < dim ? q[d] - p[d] * f : 0);
            }
      }
    }
  }
  // device lists (one allocation), then the transfers on the new stream
  // once the old stream is idle
  std::vector<int> all;
  auto put = [&](const std::vector<int>& v) {
    const size_t off = all.size();
    all.insert(all.end(), v.begin(), v.end());
    return off;
  };
  const size_t o_cto = put(cto), o_cfrom = put(cfrom), o_pf = put(pf), o_pc = put(pc), o_pld = put(pld),
               o_pidx = put(pidx), o_rf = put(rfine), o_rc = put(rcoarse), o_rld = put(rld), o_ridx = put(ridx);
  int* dl = nullptr;
  if (!salloc(&dl, std::max<size_t>(1, all.size()) * 4, nm->stream)) {
    cudaGetLastError();
    return fail(EXA_ERR_NOMEM, "exa_mesh_regrid: device allocation failed");
  }
  // frees the device lists on every return, once the new mesh's stream (which
  // reads them) is idle; declared after `guard`, so it runs before the new
  // mesh is destroyed on an error path (after the swap below the stream
  // belongs to the caller's handle and stays alive)
  struct ListGuard {
    int* p;
    cudaStream_t s;
    ~ListGuard() {
      cudaStreamSynchronize(s);
      sfree(p, s);
    }
  } dl_guard{dl, nm->stream};
  EXA_CUDA(cudaStreamSynchronize(m->stream));
  if (!all.empty()) EXA_CUDA(cudaMemcpyAsync(dl, all.data(), all.size() * 4, cudaMemcpyHostToDevice, nm->stream));
  const size_t per = (size_t)k.P * (k.nvar + k.npar);
  if (!cto.empty()) {
    copy_cells_kernel<<<std::min<size_t>((cto.size() * per + 255) / 256, 148 * 16), 256, 0, nm->stream>>>(
        nm->luh, m->luh, per, (int)cto.size(), dl + o_cto, dl + o_cfrom);
    EXA_LAUNCHED();
  }
  rc = k.amr_volume(nm->luh, m->luh, (int)pf.size(), dl + o_pf, dl + o_pc, dl + o_pld, dl + o_pidx, 0, nm->stream);
  if (!rc)
    rc = k.amr_volume(nm->luh, m->luh, (int)rfine.size(), dl + o_rf, dl + o_rc, dl + o_rld, dl + o_ridx, 1,
                      nm->stream);
  if (!rc && cudaMemcpyAsync(nm->scal, m->scal, 8 * 8, cudaMemcpyDeviceToDevice, nm->stream) != cudaSuccess)
    rc = fail(EXA_ERR_CUDA, "exa_mesh_regrid: copy failed");
  if (!rc && cudaMemcpyAsync(nm->sweeps, m->sweeps, 8, cudaMemcpyDeviceToDevice, nm->stream) != cudaSuccess)
    rc = fail(EXA_ERR_CUDA, "exa_mesh_regrid: copy failed");
  if (!rc) {  // the new admissible step from the transferred solution, then the predictor
    level_reset_kernel<<<1, 1, 0, nm->stream>>>(nm->ref.lv, nm->ref.nlev);
    EXA_LAUNCHED();
    rc = k.corrector(nm->luh, nullptr, nullptr, nullptr, mesh_dt_min(nm), nm->geo, nm->ncells, nullptr, 0, nullptr,
                     nm->stream);
  }
  if (!rc) {
    level_take_kernel<<<1, 1, 0, nm->stream>>>(nm->scal, nm->ref.lv, nm->ref.nlev);
    EXA_LAUNCHED();
    rc = mesh_predict(nm);
  }
  cudaStreamSynchronize(nm->stream);  // the old arrays are read until here
  if (rc) return rc;
  nm->initialised = true;
  // the per-phase times: the old mesh's pending events folded into its
  // totals, which carry over to the new mesh (regridding does not reset them)
  if ((rc = exa_mesh_phase_times(m, nullptr, nullptr, 0))) return rc;
  nm->profiling = m->profiling;
  for (int i = 0; i < 4; i++) {
    nm->phase_ms[i] = m->phase_ms[i];
    nm->phase_launches[i] = m->phase_launches[i];
  }
  std::swap(*m, *nm);  // the caller's handle now holds the new mesh; the guard frees the old one
  return EXA_OK;
}

int exa_mesh_run_until(exa_mesh* m, double t_end, int max_steps, int* steps) {
  if (!m) return fail(EXA_ERR_ARG, "exa_mesh_run_until: null mesh");
  if (!m->initialised) return fail(EXA_ERR_STATE, "exa_mesh_run_until: call exa_mesh_init first");
  int n = 0;
  while (n < max_steps) {
    double t, dt;
    int rc = exa_mesh_state(m, &t, &dt, nullptr, nullptr);
    if (rc) return rc;
    if (!(t < t_end && dt > 0.0)) break;
    rc = mesh_one_step(m);
    if (rc) return rc;
    n++;
  }
  if (steps) *steps = n;
  return EXA_OK;
}

int exa_mesh_stream(exa_mesh* m, void** stream) {
  if (!m || !stream) return fail(EXA_ERR_ARG, "exa_mesh_stream: null argument");
  *stream = (void*)m->stream;
  return EXA_OK;
}

int exa_mesh_set_profiling(exa_mesh* m, int on) {
  if (!m) return fail(EXA_ERR_ARG, "exa_mesh_set_profiling: null mesh");
  m->profiling = on != 0;
  return EXA_OK;
}

int exa_mesh_phase_times(exa_mesh* m, double* ms4, long long* launches4, int reset) {
  if (!m) return fail(EXA_ERR_ARG, "exa_mesh_phase_times: null mesh");
  EXA_CUDA(cudaStreamSynchronize(m->stream));
  for (size_t i = 0; i < m->ev_phase.size(); i++) {
    float ms = 0.f;
    EXA_CUDA(cudaEventElapsedTime(&ms, m->ev[2 * i], m->ev[2 * i + 1]));
    m->phase_ms[m->ev_phase[i]] += ms;
    cudaEventDestroy(m->ev[2 * i]);
    cudaEventDestroy(m->ev[2 * i + 1]);
  }
  m->ev.clear();
  m->ev_phase.clear();
  for (int i = 0; i < 4; i++) {
    if (ms4) ms4[i] = m->phase_ms[i];
    if (launches4) launches4[i] = m->phase_launches[i];
    if (reset) {
      m->phase_ms[i] = 0;
      m->phase_launches[i] = 0;
    }
  }
  return EXA_OK;
}

// best of 5 timed launches of a throughput probe on every SM (8 blocks of 256
// threads each); returns the best time in ms
}  // extern "C"
template <class Launch>
static int fp64_probe_best_ms(const char* who, Launch launch, float* best_ms) {
  double* out = nullptr;
  EXA_CUDA(cudaMalloc(&out, 8));
  cudaStream_t st;
  EXA_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  launch(out, st, true);  // warm-up
  float best = 1e30f;
  for (int r = 0; r < 5; r++) {
    cudaEventRecord(a, st);
    launch(out, st, false);
    cudaEventRecord(b, st);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (ms < best) best = ms;
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaStreamDestroy(st);
  cudaFree(out);
  if (e != cudaSuccess) return fail(EXA_ERR_CUDA, std::string(who) + ": " + cudaGetErrorString(e));
  *best_ms = best;
  return EXA_OK;
}
extern "C" {

int exa_fp64_peak_probe(double* tflops) {
  if (!tflops) return fail(EXA_ERR_ARG, "exa_fp64_peak_probe: null argument");
  int dev = 0, sms = 0;
  EXA_CUDA(cudaGetDevice(&dev));
  EXA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * 8, threads = 256, iters = 1 << 14;
  float best = 0;
  int rc = fp64_probe_best_ms("exa_fp64_peak_probe", [&](double* out, cudaStream_t st, bool warm) {
    fp64_probe_kernel<<<blocks, threads, 0, st>>>(out, warm ? 64 : iters, 0.999999, 1e-7);
  }, &best);
  if (rc) return rc;
  *tflops = 2.0 * 8.0 * iters * (double)blocks * threads / (best * 1e-3) / 1e12;
  return EXA_OK;
}

int exa_fp64_mma_peak_probe(double* tflops) {
  if (!tflops) return fail(EXA_ERR_ARG, "exa_fp64_mma_peak_probe: null argument");
  int dev = 0, sms = 0;
  EXA_CUDA(cudaGetDevice(&dev));
  EXA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const int blocks = sms * 8, threads = 256, iters = 1 << 12;
  float best = 0;
  int rc = fp64_probe_best_ms("exa_fp64_mma_peak_probe", [&](double* out, cudaStream_t st, bool warm) {
    fp64_mma_probe_kernel<<<blocks, threads, 0, st>>>(out, warm ? 16 : iters, 0.999999, 1e-7);
  }, &best);
  if (rc) return rc;
  *tflops = 2.0 * 256.0 * 4.0 * iters * ((double)blocks * threads / 32) / (best * 1e-3) / 1e12;
  return EXA_OK;
}

int exa_mesh_set_priority(exa_mesh* m, int level) {
  if (!m || level < 0) return fail(EXA_ERR_ARG, "exa_mesh_set_priority: bad argument");
  int lo = 0, hi = 0;
  EXA_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  // level 0 is the default (least) priority; greater levels are more urgent
  const int prio = std::max(hi, lo - level);
  cudaStream_t st = nullptr;
  EXA_CUDA(cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio));
  EXA_CUDA(cudaStreamSynchronize(m->stream));  // all work and allocations so far are done
  cudaStreamDestroy(m->stream);
  m->stream = st;
  return EXA_OK;
}

int exa_mesh_synchronize(exa_mesh* m) {
  if (!m) return fail(EXA_ERR_ARG, "exa_mesh_synchronize: null mesh");
  EXA_CUDA(cudaStreamSynchronize(m->stream));
  return EXA_OK;
}

}  // extern "C"

// legacy-VTK writer of exa_mesh_write_vtk: text, or binary with big-endian values
namespace {
struct VtkOut {
  FILE* f;
  bool bin;
  template <class T>
  void put(T v) {
    if (!bin) return;
    unsigned char b[sizeof(T)], r[sizeof(T)];
    std::memcpy(b, &v, sizeof(T));
    for (size_t i = 0; i < sizeof(T); i++) r[i] = b[sizeof(T) - 1 - i];
    std::fwrite(r, 1, sizeof(T), f);
  }
  void num(double v, const char* sep) {
    if (bin)
      put(v);
    else
      std::fprintf(f, "%.17g%s", v, sep);
  }
  void inum(int v, const char* sep) {
    if (bin)
      put((int32_t)v);
    else
      std::fprintf(f, "%d%s", v, sep);
  }
  void eol() {
    if (bin) std::fputc('\n', f);
  }
};
}  // namespace

extern "C" {

// legendre == 0: ADERDG2CartesianVTK (the solution projected to the (N+1)^d
// equidistant vertices of every cell); legendre != 0: ADERDG2LegendreVTK
// (exahype/plotters/VTK/ADERDG2LegendreVTK.cpp:280-380: the nodal values at
// the Gauss-Legendre nodes, offset + (cell + x_i) dx, no projection). Both
// connect the (N+1)^d points of a cell by N^d pixels / voxels.
static int mesh_write_vtk(exa_mesh* m, const char* path, int binary, int legendre, const char* fn,
                          const int* status_dev = nullptr) {
  if (!m || !path) return fail(EXA_ERR_ARG, std::string(fn) + ": null argument");
  const KernelSet& k = m->s->k;
  const int dim = m->dim, N = k.order, b = N + 1, nD = k.nvar + k.npar;
  const size_t n = m->ncells, P = k.P, sub = dim == 3 ? (size_t)N * N * N : (size_t)N * N;
  double* dev = nullptr;
  if (!legendre && !salloc(&dev, n * P * nD * 8, m->stream)) {
    cudaGetLastError();
    return fail(EXA_ERR_NOMEM, std::string(fn) + ": device allocation failed");
  }
  std::vector<double> v(n * P * nD);
  double t = 0.0;
  int rc = legendre ? EXA_OK : k.plot(m->luh, dev, (int)n, m->stream);
  if (!rc && cudaMemcpyAsync(v.data(), legendre ? m->luh : dev, v.size() * 8, cudaMemcpyDeviceToHost, m->stream) !=
                 cudaSuccess)
    rc = fail(EXA_ERR_CUDA, std::string(fn) + ": copy failed");
  if (!rc && cudaMemcpyAsync(&t, m->scal + 2, 8, cudaMemcpyDeviceToHost, m->stream) != cudaSuccess)
    rc = fail(EXA_ERR_CUDA, std::string(fn) + ": copy failed");
  std::vector<int> status(status_dev ? n : 0);
  if (!rc && status_dev &&
      cudaMemcpyAsync(status.data(), status_dev, n * 4, cudaMemcpyDeviceToHost, m->stream) != cudaSuccess)
    rc = fail(EXA_ERR_CUDA, std::string(fn) + ": copy failed");
  if (dev) sfree(dev, m->stream);
  if (rc) return rc;
  EXA_CUDA(cudaStreamSynchronize(m->stream));
  FILE* f = std::fopen(path, binary ? "wb" : "w");
  if (!f) return fail(EXA_ERR_ARG, std::string(fn) + ": cannot open " + path);
  VtkOut o{f, binary != 0};
  std::fprintf(f, "# vtk DataFile Version 3.0\nexahype_b200 ADER-DG solution t=%.17g\n%s\nDATASET UNSTRUCTURED_GRID\n",
               t, binary ? "BINARY" : "ASCII");
  // every cell is a patch of b^d vertices at offset + (cell + xi) dx, x
  // fastest, xi = i/N (equidistant) or the i-th Gauss-Legendre node
  double xi[16];
  for (int i = 0; i < b; i++) xi[i] = legendre ? exa_tab_nodes[exa_tab_nodes_off[N] + i] : (double)i / N;
  std::fprintf(f, "POINTS %zu double\n", n * P);
  for (size_t c = 0; c < n; c++) {
    // the cell's grid position and widths (its level's on a refined mesh)
    size_t cp[3] = {c % m->cells[0], (c / m->cells[0]) % m->cells[1], c / ((size_t)m->cells[0] * m->cells[1])};
    const double* w = m->geo.dx;
    if (m->ref.on) {
      for (int d = 0; d < 3; d++) cp[d] = (size_t)m->ref.pos[3 * c + d];
      w = &m->ref.ldx[3 * (size_t)m->ref.level[c]];
    }
    for (size_t p = 0; p < P; p++) {
      const int ix = (int)(p % b), iy = (int)((p / b) % b), iz = dim == 3 ? (int)(p / (b * b)) : 0;
      o.num(m->offset[0] + (cp[0] + xi[ix]) * w[0], " ");
      o.num(m->offset[1] + (cp[1] + xi[iy]) * w[1], " ");
      o.num(dim == 3 ? m->offset[2] + (cp[2] + xi[iz]) * w[2] : 0.0, "\n");
    }
  }
  o.eol();
  const int nv = dim == 3 ? 8 : 4;
  std::fprintf(f, "CELLS %zu %zu\n", n * sub, n * sub * (nv + 1));
  for (size_t c = 0; c < n; c++)
    for (int kz = 0; kz < (dim == 3 ? N : 1); kz++)
      for (int ky = 0; ky < N; ky++)
        for (int kx = 0; kx < N; kx++) {
          o.inum(nv, " ");
          // VTK_PIXEL / VTK_VOXEL vertex order: x fastest, then y, then z
          for (int q = 0; q < nv; q++) {
            const int dx = q & 1, dy = (q >> 1) & 1, dz = (q >> 2) & 1;
            const size_t id = c * P + ((size_t)(kz + dz) * b + (ky + dy)) * b + (kx + dx);
            o.inum((int)id, q + 1 < nv ? " " : "\n");
          }
        }
  o.eol();
  std::fprintf(f, "CELL_TYPES %zu\n", n * sub);
  for (size_t i = 0; i < n * sub; i++) o.inum(dim == 3 ? 11 : 8, "\n");
  o.eol();
  std::fprintf(f, "POINT_DATA %zu\nSCALARS Q double %d\nLOOKUP_TABLE default\n", n * P, nD);
  for (size_t i = 0; i < n * P; i++)
    for (int q = 0; q < nD; q++) o.num(v[i * nD + q], q + 1 < nD ? " " : "\n");
  o.eol();
  std::fprintf(f, "SCALARS time double 1\nLOOKUP_TABLE default\n");
  for (size_t i = 0; i < n * P; i++) o.num(t, "\n");
  o.eol();
  if (status_dev) {  // LimitingADERDG2CartesianVTK's vertex "Limiter-Status" (the cell's status)
    std::fprintf(f, "SCALARS Limiter-Status double 1\nLOOKUP_TABLE default\n");
    for (size_t i = 0; i < n * P; i++) o.num((double)status[i / P], "\n");
    o.eol();
  }
  const bool ok = std::ferror(f) == 0;
  std::fclose(f);
  if (!ok) return fail(EXA_ERR_ARG, std::string(fn) + ": write error on " + path);
  return EXA_OK;
}

int exa_mesh_write_vtk(exa_mesh* m, const char* path, int binary) {
  return mesh_write_vtk(m, path, binary, 0, "exa_mesh_write_vtk");
}

int exa_mesh_write_vtk_legendre(exa_mesh* m, const char* path, int binary) {
  return mesh_write_vtk(m, path, binary, 1, "exa_mesh_write_vtk_legendre");
}

}  // extern "C"

// ---- limiting mesh ------------------------------------------------------------
struct exa_lmesh {
  exa_mesh* m = nullptr;  // DG state, faces, stream and time scalars
  int A = 2, T = 3, cure_steps = 0;
  double relax = 1e-4, scale = 1e-3;
  // s: limiter status; flags: [0] irregular change this step, [1] DG list
  // length, [2] FV list length, [3] predictor list length, [4] run flag of
  // run_until's captured step
  int *s = nullptr, *s_prev = nullptr, *cure = nullptr, *fs = nullptr, *has_lim = nullptr, *flags = nullptr;
  int *listA = nullptr, *listF = nullptr, *listP = nullptr;
  double *minB = nullptr, *maxB = nullptr, *lim = nullptr, *lim_prev = nullptr, *luh_prev = nullptr;
  double *fv_ic = nullptr, *gscratch = nullptr;
  int muscl_grid = 1;
  size_t LS = 0, PB = 0;  // doubles per FV patch (ghosts included), subcells per cell
  int (*init)(exa_lmesh*, double) = nullptr;
  int (*step)(exa_lmesh*) = nullptr;
  int (*chunk)(exa_lmesh*, int) = nullptr;
  cudaGraphExec_t graph = nullptr;  // captured gated step of run_until
  int graph_variant = -1;
  bool initialised = false;
};

namespace exa {

// scal: [0] dt, [1] min target after the update, [2] t, [3] steps,
//       [4] min target after a local recomputation, [5] irregular steps,
//       [6] end time of run_until
__global__ void lim_scalars_kernel(double* scal, double t0) {
  scal[0] = 0.0;
  scal[1] = __longlong_as_double(0x7fefffffffffffffll);
  scal[2] = t0;
  scal[3] = 0.0;
  scal[4] = __longlong_as_double(0x7fefffffffffffffll);
  scal[5] = 0.0;
}

// Time bookkeeping of a limiting step: on an irregular step the reference's
// LocalRecomputation::endIteration runs startNewTimeStep() once more
// (mappings/LocalRecomputation.cpp:193-207 after SolutionUpdate.cpp:308-322),
// so the time stamp also advances by the step found after the update, and the
// next step uses the one found after the recomputation.
__global__ void lim_advance_kernel(double* scal, const int* flags, const int* run) {
  if (run && !*run) return;
  const bool irr = flags[0] != 0;
  scal[2] += scal[0];
  if (irr) scal[2] += scal[1];
  scal[0] = irr ? scal[4] : scal[1];
  scal[1] = __longlong_as_double(0x7fefffffffffffffll);
  scal[4] = __longlong_as_double(0x7fefffffffffffffll);
  scal[3] += 1.0;
  if (irr) scal[5] += 1.0;
}

// run flag of the next step of run_until: t < t_end (scal[6]) and dt > 0
__global__ void lim_run_gate_kernel(const double* scal, int* run) { *run = scal[2] < scal[6] && scal[0] > 0.0; }

template <int DIM, int N>
struct LimLaunch {
  using PDE = EulerPDE;
  using L = LimShape<DIM, N>;
  using MC = MusclCfg<DIM, N>;
  using PC = PostCfg<DIM, N>;
  static constexpr int PROJ_TMP = tensor_tmp<DIM, L::b, L::B>() > tensor_tmp<DIM, L::B, L::b>()
                                      ? tensor_tmp<DIM, L::b, L::B>() : tensor_tmp<DIM, L::B, L::b>();
  static constexpr size_t PROJ_SMEM = sizeof(double) * PROJ_TMP;
  static_assert(MC::SMEM <= 227 * 1024 && PC::SMEM <= 227 * 1024 && PROJ_SMEM <= 227 * 1024, "shared memory");

  static int attrs() {
    static bool done = false;
    if (done) return EXA_OK;
    EXA_CUDA(cudaFuncSetAttribute(lim_muscl_kernel<DIM, N, PDE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)MC::SMEM));
    EXA_CUDA(cudaFuncSetAttribute(lim_post_update_kernel<DIM, N, PDE, typename PC::Group>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PC::POST_SMEM));
    EXA_CUDA(cudaFuncSetAttribute(lim_init_kernel<DIM, N, PDE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)PC::SMEM));
    EXA_CUDA(cudaFuncSetAttribute(lim_seed_kernel<DIM, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)PROJ_SMEM));
    EXA_CUDA(cudaFuncSetAttribute(lim_reinit_kernel<DIM, N, typename PC::Group>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(PROJ_SMEM * PC::CELLS)));
    EXA_CUDA(cudaFuncSetAttribute(lim_recompute_kernel<DIM, N, PDE, typename PC::Group>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(PROJ_SMEM * PC::CELLS)));
    EXA_CUDA(cudaFuncSetAttribute(lim_project_kernel<DIM, N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)PROJ_SMEM));
    done = true;
    return EXA_OK;
  }
  // MUSCL blocks resident on the device at once (grid-stride over the FV list)
  static int muscl_grid(int ncells, int* grid) {
    EXA_CUDA(cudaFuncSetAttribute(lim_muscl_kernel<DIM, N, PDE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)MC::SMEM));
    int dev = 0, sms = 0, per_sm = 0;
    EXA_CUDA(cudaGetDevice(&dev));
    EXA_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    EXA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, lim_muscl_kernel<DIM, N, PDE>, MC::THREADS,
                                                           MC::SMEM));
    *grid = std::max(1, std::min(ncells, sms * std::max(1, per_sm)));
    return EXA_OK;
  }
  static size_t scratch_doubles() { return MC::kShared ? 0 : (size_t)MC::SCR; }

  // kernel-level entry points (no mesh): MUSCL-Hancock over a cell list with
  // caller-provided scratch, and the two projections
  static int muscl_call(double* lim, double* lim_old, double* luh, const double* dt, Geometry g, int n,
                        const int* list, double* scratch, size_t scratch_doubles_avail, cudaStream_t st) {
    if (n <= 0) return EXA_OK;
    int rc = attrs();
    if (rc) return rc;
    int grid = 0;
    if ((rc = muscl_grid(n, &grid))) return rc;
    if (!MC::kShared) {
      const size_t fit = scratch_doubles_avail / (size_t)MC::SCR;
      if (fit < 1 || !scratch)
        return fail(EXA_ERR_ARG, "exa_fv_musclhancock_update: scratch holds " +
                                     std::to_string(scratch_doubles_avail * 8) + " bytes, one block needs " +
                                     std::to_string((size_t)MC::SCR * 8));
      grid = (int)std::min<size_t>((size_t)grid, fit);
    }
    lim_muscl_kernel<DIM, N, PDE><<<grid, MC::THREADS, MC::SMEM, st>>>(list, nullptr, n, lim, lim_old, luh, g, dt,
                                                                       scratch, nullptr);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static int scratch_bytes_for(int n, size_t* bytes) {
    if (MC::kShared || n <= 0) {
      *bytes = 0;
      return EXA_OK;
    }
    int grid = 0;
    int rc = muscl_grid(n, &grid);
    if (rc) return rc;
    *bytes = (size_t)grid * MC::SCR * sizeof(double);
    return EXA_OK;
  }
  static int project_call(double* luh, double* lim, int n, const int* list, int to_fv, cudaStream_t st) {
    if (n <= 0) return EXA_OK;
    int rc = attrs();
    if (rc) return rc;
    lim_project_kernel<DIM, N><<<n, 128, PROJ_SMEM, st>>>(list, n, luh, lim, to_fv);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static LimParams params(const exa_lmesh* lm) { return LimParams{lm->A, lm->T, lm->cure_steps, lm->relax, lm->scale}; }

  static int select(exa_lmesh* lm, int lo, int hi, int* list, int* count, const int* gate) {
    exa_mesh* m = lm->m;
    EXA_CUDA(cudaMemsetAsync(count, 0, sizeof(int), m->stream));
    lim_select_kernel<<<(m->ncells + 255) / 256, 256, 0, m->stream>>>(m->ncells, lm->s, lo, hi, list, count, gate);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static int merge(exa_lmesh* lm, int minmax, const int* gate) {
    exa_mesh* m = lm->m;
    if (m->nfaces <= 0) return EXA_OK;
    lim_merge_faces_kernel<DIM><<<(m->nfaces + 127) / 128, 128, 0, m->stream>>>(
        m->fl, m->fr, m->fd, m->nfaces, lm->s, lm->minB, lm->maxB, lm->fs, lm->T, minmax, gate);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static int spread(exa_lmesh* lm, const int* gate) {  // T sweeps of limiter status spreading
    exa_mesh* m = lm->m;
    for (int it = 0; it < lm->T; it++) {
      int rc = merge(lm, 0, gate);
      if (rc) return rc;
      lim_spread_cells_kernel<DIM, N><<<(m->ncells + 3) / 4, 128, 0, m->stream>>>(
          m->ncells, lm->s, lm->cure, lm->fs, lm->has_lim, lm->lim, lm->lim_prev, params(lm), gate);
      EXA_LAUNCHED();
    }
    return EXA_OK;
  }
  static int halo(exa_lmesh* lm, const int* gate) {  // boundary faces: outflow, then reflective (grouped)
    exa_mesh* m = lm->m;
    const int nb0 = m->nbfaces[EXA_BC_OUTFLOW], nb = nb0 + m->nbfaces[EXA_BC_REFLECTIVE], total = m->nfaces + nb;
    if (total <= 0) return EXA_OK;
    lim_fv_halo_kernel<DIM, N><<<(total + 3) / 4, 128, 0, m->stream>>>(
        m->fl, m->fr, m->fd, m->nfaces, m->bcell, m->bface, nb, nb0, lm->s, lm->has_lim, lm->lim, lm->A, gate);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static int muscl(exa_lmesh* lm, const int* gate) {
    exa_mesh* m = lm->m;
    lim_muscl_kernel<DIM, N, PDE><<<lm->muscl_grid, MC::THREADS, MC::SMEM, m->stream>>>(
        lm->listF, lm->flags + 2, 0, lm->lim, lm->lim_prev, m->luh, m->geo, m->scal + 0, lm->gscratch, gate);
    EXA_LAUNCHED();
    return EXA_OK;
  }
  static int predict(exa_lmesh* lm, const int* run = nullptr) {  // status < T (mappings/Prediction.cpp:176-178)
    exa_mesh* m = lm->m;
    int rc = select(lm, INT_MIN, lm->T, lm->listP, lm->flags + 3, run);
    if (rc) return rc;
    return m->s->k.predictor(m->luh, m->lQhbnd, m->lFhbnd, m->lduh, m->iters, m->scal + 0, m->geo, m->ncells,
                             lm->listP, lm->flags + 3, PredictorTemps{}, false, m->sweeps, m->s->variant, m->stream);
  }

  static int init(exa_lmesh* lm, double t0) {
    exa_mesh* m = lm->m;
    const int n = m->ncells;
    int rc = attrs();
    if (rc) return rc;
    lim_scalars_kernel<<<1, 1, 0, m->stream>>>(m->scal, t0);
    EXA_LAUNCHED();
    EXA_CUDA(cudaMemsetAsync(m->sweeps, 0, 8, m->stream));
    EXA_CUDA(cudaMemsetAsync(lm->flags, 0, 4 * sizeof(int), m->stream));
    lim_init_kernel<DIM, N, PDE><<<n, PC::THREADS, PC::SMEM, m->stream>>>(
        n, m->luh, lm->s, lm->s_prev, lm->cure, lm->fs, lm->has_lim, lm->minB, lm->maxB, params(lm));
    EXA_LAUNCHED();
    if ((rc = spread(lm, nullptr))) return rc;
    lim_seed_kernel<DIM, N><<<n, 128, PROJ_SMEM, m->stream>>>(n, lm->s, m->luh, lm->fv_ic, lm->lim);
    EXA_LAUNCHED();
    if ((rc = m->s->k.corrector(m->luh, nullptr, nullptr, nullptr, m->scal + 1, m->geo, n, nullptr, 0, nullptr,
                                m->stream)))
      return rc;
    take_dt_kernel<<<1, 1, 0, m->stream>>>(m->scal);
    EXA_LAUNCHED();
    return predict(lm);
  }

  // One limiting step. run (optional, device): when it holds 0 every launch
  // of the step returns at once (run_until replays captured steps past t_end).
  static int step_launch(exa_lmesh* lm, const int* run) {
    exa_mesh* m = lm->m;
    const KernelSet& k = m->s->k;
    const int n = m->ncells;
    const LimParams prm = params(lm);
    cudaStream_t st = m->stream;
    int rc;
    EXA_CUDA(cudaMemsetAsync(lm->flags, 0, sizeof(int), st));
    // merge: DMP min/max and facewise statuses; DG Riemann problems (the
    // fluxes of faces between two FV-active cells are computed but never
    // read); FV halo exchange and FV boundary on FV-active faces
    if ((rc = merge(lm, 1, run))) return rc;
    if ((rc = k.riemann(m->lQhbnd, m->lFhbnd, m->fl, m->fr, m->fd, m->nfaces, run, st))) return rc;
    for (int kd : {EXA_BC_OUTFLOW, EXA_BC_REFLECTIVE})
      if ((rc = k.boundary(m->lQhbnd, m->lFhbnd, m->bcell + m->boff[kd], m->bface + m->boff[kd], m->nbfaces[kd], kd,
                           run, st)))
        return rc;
    if ((rc = halo(lm, run))) return rc;
    // update: DG cells (s < A) by the corrector, FV-active cells by
    // MUSCL-Hancock (lists come out empty when run holds 0)
    EXA_CUDA(cudaMemcpyAsync(lm->luh_prev, m->luh, (size_t)n * L::P * L::nV * sizeof(double),
                             cudaMemcpyDeviceToDevice, st));
    // both lists from the statuses before the update (the corrector does not
    // change them); counters flags[1], flags[2]
    EXA_CUDA(cudaMemsetAsync(lm->flags + 1, 0, 2 * sizeof(int), st));
    lim_select2_kernel<<<(n + 255) / 256, 256, 0, st>>>(n, lm->s, INT_MIN, lm->A, lm->listA, lm->flags + 1, lm->A,
                                                        INT_MAX, lm->listF, lm->flags + 2, run);
    EXA_LAUNCHED();
    if ((rc = k.corrector(m->luh, m->lduh, m->lFhbnd, m->scal + 0, nullptr, m->geo, n, lm->listA, 1, lm->flags + 1,
                          st)))
      return rc;
    if ((rc = muscl(lm, run))) return rc;
    lim_post_update_kernel<DIM, N, PDE, typename PC::Group>
        <<<(n + PC::CELLS - 1) / PC::CELLS, PC::THREADS, PC::POST_SMEM, st>>>(
        n, m->luh, lm->s, lm->s_prev, lm->cure, lm->fs, lm->has_lim, lm->minB, lm->maxB, lm->lim, lm->lim_prev,
        m->geo, prm, m->scal + 1, lm->flags, run);
    EXA_LAUNCHED();
    // irregular limiter domain change: every launch below returns at once
    // unless the post-update kernel raised flags[0] (it never does on a step
    // that run skips)
    const int* g = lm->flags;
    if ((rc = spread(lm, g))) return rc;
    lim_reinit_kernel<DIM, N, typename PC::Group><<<(n + PC::CELLS - 1) / PC::CELLS, 128, PROJ_SMEM * PC::CELLS, st>>>(
        n, m->luh, lm->luh_prev, lm->s, lm->s_prev, lm->cure,
                                                          lm->has_lim, lm->lim, lm->lim_prev, prm, g);
    EXA_LAUNCHED();
    if ((rc = halo(lm, g))) return rc;
    if ((rc = select(lm, lm->A, INT_MAX, lm->listF, lm->flags + 2, g))) return rc;
    if ((rc = muscl(lm, g))) return rc;
    lim_recompute_kernel<DIM, N, PDE, typename PC::Group>
        <<<(n + PC::CELLS - 1) / PC::CELLS, 128, PROJ_SMEM * PC::CELLS, st>>>(n, m->luh, lm->luh_prev, lm->s, lm->s_prev,
                                                                  lm->lim, lm->lim_prev, m->geo, prm, m->scal + 4, g);
    EXA_LAUNCHED();
    lim_advance_kernel<<<1, 1, 0, st>>>(m->scal, lm->flags, run);
    EXA_LAUNCHED();
    return predict(lm, run);
  }
  static int step(exa_lmesh* lm) { return step_launch(lm, nullptr); }

  // k steps of run_until: the step is captured once as a CUDA graph whose
  // first node sets the run flag (t < t_end && dt > 0, t_end in scal[6]) and
  // is replayed k times; replays past t_end change nothing.
  static int chunk(exa_lmesh* lm, int k) {
    cudaStream_t st = lm->m->stream;
    if (!lm->graph || lm->graph_variant != lm->m->s->variant) {
      if (lm->graph) {
        EXA_CUDA(cudaStreamSynchronize(st));
        cudaGraphExecDestroy(lm->graph);
      }
      lm->graph = nullptr;
      cudaGraph_t g = nullptr;
      EXA_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      lim_run_gate_kernel<<<1, 1, 0, st>>>(lm->m->scal, lm->flags + 4);
      const int rc = step_launch(lm, lm->flags + 4);
      const cudaError_t e = cudaStreamEndCapture(st, &g);
      if (rc || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return rc ? rc : fail(EXA_ERR_CUDA, std::string("exa_lmesh_run_until: capture: ") + cudaGetErrorString(e));
      }
      const cudaError_t e2 = cudaGraphInstantiate(&lm->graph, g, 0);
      cudaGraphDestroy(g);
      if (e2 != cudaSuccess) {
        lm->graph = nullptr;
        return fail(EXA_ERR_CUDA, std::string("exa_lmesh_run_until: instantiate: ") + cudaGetErrorString(e2));
      }
      lm->graph_variant = lm->m->s->variant;
    }
    for (int i = 0; i < k; i++) EXA_CUDA(cudaGraphLaunch(lm->graph, st));
    return EXA_OK;
  }
};

struct LimOps {
  int (*init)(exa_lmesh*, double);
  int (*step)(exa_lmesh*);
  int (*chunk)(exa_lmesh*, int);
  int (*grid)(int, int*);
  size_t (*scratch)();
  size_t LS, PB;
  int (*muscl)(double*, double*, double*, const double*, Geometry, int, const int*, double*, size_t, cudaStream_t);
  int (*scratch_bytes)(int, size_t*);
  int (*project)(double*, double*, int, const int*, int, cudaStream_t);
};

static bool find_lim_ops(int dim, int order, LimOps* out) {
#define X(D, NN, PDE_, ID)                                                                              \
  if (dim == D && order == NN) {                                                                        \
    using LL = LimLaunch<D, NN>;                                                                        \
    *out = LimOps{&LL::init, &LL::step, &LL::chunk, &LL::muscl_grid, &LL::scratch_doubles, (size_t)LimShape<D, NN>::LS, \
                  (size_t)LimShape<D, NN>::PB, &LL::muscl_call, &LL::scratch_bytes_for, &LL::project_call};   \
    return true;                                                                                        \
  }
  EXA_ORDERS_EULER(X, 2)
  EXA_ORDERS_EULER(X, 3)
#undef X
  return false;
}

}  // namespace exa

extern "C" {

static int lim_ops_of(const exa_solver* s, const char* fn, LimOps* ops) {
  if (!s) return fail(EXA_ERR_ARG, std::string(fn) + ": null solver");
  if (s->k.pde != EXA_PDE_EULER) return fail(EXA_ERR_UNSUPPORTED, std::string(fn) + ": the limiter supports EXA_PDE_EULER");
  if (!find_lim_ops(s->k.dim, s->k.order, ops))
    return fail(EXA_ERR_UNSUPPORTED, std::string(fn) + ": no limiter kernels for this order");
  return EXA_OK;
}

int exa_project_on_fv_limiter_space(const exa_solver* s, const double* luh, double* lim, int ncells,
                                    const int* cell_list, void* stream) {
  LimOps ops;
  int rc = lim_ops_of(s, "exa_project_on_fv_limiter_space", &ops);
  if (rc) return rc;
  if (!luh || !lim || ncells < 0) return fail(EXA_ERR_ARG, "exa_project_on_fv_limiter_space: bad argument");
  return ops.project(const_cast<double*>(luh), lim, ncells, cell_list, 1, (cudaStream_t)stream);
}

int exa_project_on_dg_space(const exa_solver* s, const double* lim, double* luh, int ncells, const int* cell_list,
                            void* stream) {
  LimOps ops;
  int rc = lim_ops_of(s, "exa_project_on_dg_space", &ops);
  if (rc) return rc;
  if (!luh || !lim || ncells < 0) return fail(EXA_ERR_ARG, "exa_project_on_dg_space: bad argument");
  return ops.project(luh, const_cast<double*>(lim), ncells, cell_list, 0, (cudaStream_t)stream);
}

int exa_fv_musclhancock_scratch_bytes(const exa_solver* s, int ncells, size_t* bytes) {
  LimOps ops;
  int rc = lim_ops_of(s, "exa_fv_musclhancock_scratch_bytes", &ops);
  if (rc) return rc;
  if (!bytes || ncells < 0) return fail(EXA_ERR_ARG, "exa_fv_musclhancock_scratch_bytes: bad argument");
  return ops.scratch_bytes(ncells, bytes);
}

int exa_fv_musclhancock_update(const exa_solver* s, double* lim, double* lim_old, double* luh, const double* dt_dev,
                               const double* dx, int ncells, const int* cell_list, void* scratch, size_t scratch_bytes,
                               void* stream) {
  LimOps ops;
  int rc = lim_ops_of(s, "exa_fv_musclhancock_update", &ops);
  if (rc) return rc;
  if (!lim || !lim_old || !dt_dev || !dx || ncells < 0)
    return fail(EXA_ERR_ARG, "exa_fv_musclhancock_update: bad argument");
  return ops.muscl(lim, lim_old, luh, dt_dev, geom(s, dx), ncells, cell_list, (double*)scratch,
                   scratch_bytes / sizeof(double), (cudaStream_t)stream);
}

// ---- MUSCL-Hancock without device allocation ---------------------------------
// exa_fv_musclhancock_update_noalloc runs the same kernel as
// exa_fv_musclhancock_update with the library's own scratch: a file-scope
// __device__ array of kNoAllocScratchBytes, found once per device by
// cudaGetSymbolAddress. The call allocates nothing. Nothing in the array needs
// to start at zero (every slot a block reads was written by that block for the
// same cell). Calls that overlap in time share the array and race.
constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double)];

// The current context of the calling thread (the device's primary context
// once the runtime has touched it), through the driver entry point the
// runtime exposes, so that the library needs no link against the driver.
static void* current_context() {
  typedef int (*CtxGetCurrent)(void**);
  static CtxGetCurrent fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<CtxGetCurrent>(f);
  }();
  void* ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

// The device address of g_noalloc_scratch for the current device, looked up
// with cudaGetSymbolAddress on the first call per device and context (the
// host-side name of the array is no device address) and cached under the
// context it was found in: after a reset of the device the module is loaded
// into a new primary context and the address is looked up again.
static int noalloc_scratch(double** out) {
  static std::mutex mu;
  struct Entry {
    int dev;
    void* ctx;
    double* p;
  };
  static std::vector<Entry> per_device;
  int dev = 0;
  EXA_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  void* ctx = current_context();
  for (const auto& e : per_device)
    if (e.dev == dev && e.ctx == ctx && ctx) {
      *out = e.p;
      return EXA_OK;
    }
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return fail(EXA_ERR_CUDA, std::string("exa_fv_musclhancock_update_noalloc: cudaGetSymbolAddress: ") +
                                  cudaGetErrorString(e));
  ctx = current_context();  // the lookup makes the runtime's context current if it was not yet
  for (auto& en : per_device)
    if (en.dev == dev) {
      en.ctx = ctx;
      en.p = static_cast<double*>(p);
      *out = en.p;
      return EXA_OK;
    }
  per_device.push_back(Entry{dev, ctx, static_cast<double*>(p)});
  *out = static_cast<double*>(p);
  return EXA_OK;
}

int exa_fv_musclhancock_update_noalloc(const exa_solver* s, double* lim, double* lim_old, double* luh,
                                       const double* dt_dev, const double* dx, int ncells, const int* cell_list,
                                       void* stream) {
  LimOps ops;
  int rc = lim_ops_of(s, "exa_fv_musclhancock_update_noalloc", &ops);
  if (rc) return rc;
  if (!lim || !lim_old || !dt_dev || !dx || ncells < 0)
    return fail(EXA_ERR_ARG, "exa_fv_musclhancock_update_noalloc: bad argument");
  const size_t per_block = ops.scratch() * sizeof(double);
  if (per_block > kNoAllocScratchBytes)
    return fail(EXA_ERR_UNSUPPORTED, "exa_fv_musclhancock_update_noalloc: one block of this order needs " +
                                         std::to_string(per_block) + " bytes of scratch, the static scratch holds " +
                                         std::to_string(kNoAllocScratchBytes));
  double* scratch = nullptr;
  if (per_block > 0 && (rc = noalloc_scratch(&scratch))) return rc;
  return ops.muscl(lim, lim_old, luh, dt_dev, geom(s, dx), ncells, cell_list, scratch,
                   kNoAllocScratchBytes / sizeof(double), (cudaStream_t)stream);
}

static void lmesh_free(exa_lmesh* lm) {
  cudaStream_t st = lm->m ? lm->m->stream : nullptr;
  if (lm->graph) cudaGraphExecDestroy(lm->graph);
  lm->graph = nullptr;
  for (void* p : {(void*)lm->s, (void*)lm->s_prev, (void*)lm->cure, (void*)lm->fs, (void*)lm->has_lim,
                  (void*)lm->flags, (void*)lm->listA, (void*)lm->listF, (void*)lm->listP, (void*)lm->minB,
                  (void*)lm->maxB, (void*)lm->lim, (void*)lm->lim_prev, (void*)lm->luh_prev, (void*)lm->fv_ic,
                  (void*)lm->gscratch})
    sfree(p, st);
  if (lm->m) exa_mesh_destroy(lm->m);
  lm->m = nullptr;
}

int exa_lmesh_create(const exa_solver* s, const int* cells, const double* offset, const double* size, const int* bc,
                     int helper_layers, int cure_steps, double relax, double scale, exa_lmesh** out) {
  if (!s || !cells || !offset || !size || !bc || !out) return fail(EXA_ERR_ARG, "exa_lmesh_create: null argument");
  if (s->k.pde != EXA_PDE_EULER) return fail(EXA_ERR_UNSUPPORTED, "exa_lmesh_create: the limiter supports EXA_PDE_EULER");
  if (helper_layers < 1 || helper_layers > 8 || cure_steps < 0 || !(relax >= 0) || !(scale >= 0))
    return fail(EXA_ERR_ARG, "exa_lmesh_create: helper_layers 1..8, cure_steps >= 0, relax/scale >= 0");
  LimOps ops{};
  if (!find_lim_ops(s->k.dim, s->k.order, &ops))
    return fail(EXA_ERR_UNSUPPORTED, "exa_lmesh_create: no limiter kernels for this order");
  std::unique_ptr<exa_lmesh> lm(new exa_lmesh());
  int rc = exa_mesh_create(s, cells, offset, size, bc, &lm->m);
  if (rc) return rc;
  lm->A = helper_layers + 1;
  lm->T = 2 * helper_layers + 1;
  lm->cure_steps = cure_steps;
  lm->relax = relax;
  lm->scale = scale;
  lm->LS = ops.LS;
  lm->PB = ops.PB;
  lm->init = ops.init;
  lm->step = ops.step;
  lm->chunk = ops.chunk;
  const size_t n = lm->m->ncells, D2 = 2 * s->k.dim, P = s->k.P;
  rc = ops.grid((int)n, &lm->muscl_grid);
  if (rc) {
    lmesh_free(lm.get());
    return rc;
  }
  const size_t scr = ops.scratch();
  cudaStream_t lst = lm->m->stream;
  bool ok = salloc(&lm->s, n * 4, lst) && salloc(&lm->s_prev, n * 4, lst) && salloc(&lm->cure, n * 4, lst) &&
            salloc(&lm->fs, n * D2 * 4, lst) && salloc(&lm->has_lim, n * 4, lst) && salloc(&lm->flags, 8 * 4, lst) &&
            salloc(&lm->listA, n * 4, lst) && salloc(&lm->listF, n * 4, lst) && salloc(&lm->listP, n * 4, lst) &&
            salloc(&lm->minB, n * D2 * 5 * 8, lst) && salloc(&lm->maxB, n * D2 * 5 * 8, lst) &&
            salloc(&lm->lim, n * lm->LS * 8, lst) && salloc(&lm->lim_prev, n * lm->LS * 8, lst) &&
            salloc(&lm->luh_prev, n * P * 5 * 8, lst) &&
            (scr == 0 || salloc(&lm->gscratch, (size_t)lm->muscl_grid * scr * 8, lst));
  if (!ok) {
    cudaGetLastError();
    lmesh_free(lm.get());
    return fail(EXA_ERR_NOMEM, "exa_lmesh_create: device allocation failed");
  }
  cudaStream_t st = lm->m->stream;
  EXA_CUDA(cudaMemsetAsync(lm->s, 0, n * 4, st));
  EXA_CUDA(cudaMemsetAsync(lm->s_prev, 0, n * 4, st));
  EXA_CUDA(cudaMemsetAsync(lm->cure, 0, n * 4, st));
  EXA_CUDA(cudaMemsetAsync(lm->fs, 0, n * D2 * 4, st));
  EXA_CUDA(cudaMemsetAsync(lm->has_lim, 0, n * 4, st));
  EXA_CUDA(cudaMemsetAsync(lm->flags, 0, 32, st));
  EXA_CUDA(cudaMemsetAsync(lm->lim, 0, n * lm->LS * 8, st));
  EXA_CUDA(cudaMemsetAsync(lm->lim_prev, 0, n * lm->LS * 8, st));
  EXA_CUDA(cudaMemsetAsync(lm->luh_prev, 0, n * P * 5 * 8, st));
  EXA_CUDA(cudaStreamSynchronize(st));
  *out = lm.release();
  return EXA_OK;
}

int exa_lmesh_destroy(exa_lmesh* lm) {
  if (!lm) return EXA_OK;
  lmesh_free(lm);
  delete lm;
  return EXA_OK;
}

int exa_lmesh_set_solution(exa_lmesh* lm, const double* h) {
  if (!lm) return fail(EXA_ERR_ARG, "exa_lmesh_set_solution: null mesh");
  return exa_mesh_set_solution(lm->m, h);
}

int exa_lmesh_get_solution(exa_lmesh* lm, double* h) {
  if (!lm) return fail(EXA_ERR_ARG, "exa_lmesh_get_solution: null mesh");
  return exa_mesh_get_solution(lm->m, h);
}

int exa_lmesh_write_vtk(exa_lmesh* lm, const char* path, int binary) {
  if (!lm) return fail(EXA_ERR_ARG, "exa_lmesh_write_vtk: null mesh");
  return mesh_write_vtk(lm->m, path, binary, 0, "exa_lmesh_write_vtk", lm->s);
}

int exa_lmesh_set_fv_initial(exa_lmesh* lm, const double* h) {
  if (!lm || !h) return fail(EXA_ERR_ARG, "exa_lmesh_set_fv_initial: null argument");
  const size_t bytes = (size_t)lm->m->ncells * lm->PB * 5 * 8;
  if (!lm->fv_ic && !salloc(&lm->fv_ic, bytes, lm->m->stream)) {
    cudaGetLastError();
    lm->fv_ic = nullptr;
    return fail(EXA_ERR_NOMEM, "exa_lmesh_set_fv_initial: device allocation failed");
  }
  EXA_CUDA(cudaMemcpyAsync(lm->fv_ic, h, bytes, cudaMemcpyHostToDevice, lm->m->stream));
  EXA_CUDA(cudaStreamSynchronize(lm->m->stream));
  return EXA_OK;
}

int exa_lmesh_init(exa_lmesh* lm, double t0) {
  if (!lm) return fail(EXA_ERR_ARG, "exa_lmesh_init: null mesh");
  int rc = lm->init(lm, t0);
  if (rc) return rc;
  lm->initialised = true;
  return EXA_OK;
}

int exa_lmesh_step(exa_lmesh* lm, int nsteps) {
  if (!lm) return fail(EXA_ERR_ARG, "exa_lmesh_step: null mesh");
  if (!lm->initialised) return fail(EXA_ERR_STATE, "exa_lmesh_step: call exa_lmesh_init first");
  for (int i = 0; i < nsteps; i++) {
    int rc = lm->step(lm);
    if (rc) return rc;
  }
  return EXA_OK;
}

int exa_lmesh_state(exa_lmesh* lm, double* t, double* dt, long long* steps, long long* sweeps, long long* irregular) {
  if (!lm) return fail(EXA_ERR_ARG, "exa_lmesh_state: null mesh");
  exa_mesh* m = lm->m;
  double h[6];
  unsigned long long sw = 0;
  EXA_CUDA(cudaMemcpyAsync(h, m->scal, sizeof(h), cudaMemcpyDeviceToHost, m->stream));
  EXA_CUDA(cudaMemcpyAsync(&sw, m->sweeps, 8, cudaMemcpyDeviceToHost, m->stream));
  EXA_CUDA(cudaStreamSynchronize(m->stream));
  if (t) *t = h[2];
  if (dt) *dt = h[0];
  if (steps) *steps = (long long)h[3];
  if (sweeps) *sweeps = (long long)sw;
  if (irregular) *irregular = (long long)h[5];
  return EXA_OK;
}

int exa_lmesh_run_until(exa_lmesh* lm, double t_end, int max_steps, int* steps) {
  if (!lm) return fail(EXA_ERR_ARG, "exa_lmesh_run_until: null mesh");
  if (!lm->initialised) return fail(EXA_ERR_STATE, "exa_lmesh_run_until: call exa_lmesh_init first");
  // Steps are replayed from a captured graph in chunks of up to 16; each
  // replay runs a step only while t < t_end and dt > 0 hold on the device, so
  // the steps taken are the ones a step-by-step loop checking t on the host
  // would take. The host reads the time once per chunk.
  constexpr int kChunk = 16;
  double t = 0.0, dt = 0.0;
  long long s0 = 0, s1 = 0;
  int rc = exa_lmesh_state(lm, &t, &dt, &s0, nullptr, nullptr);
  if (rc) return rc;
  EXA_CUDA(cudaMemcpyAsync(lm->m->scal + 6, &t_end, sizeof(double), cudaMemcpyHostToDevice, lm->m->stream));
  int n = 0;
  while (n < max_steps && t < t_end && dt > 0.0) {
    if ((rc = lm->chunk(lm, std::min(kChunk, max_steps - n)))) return rc;
    if ((rc = exa_lmesh_state(lm, &t, &dt, &s1, nullptr, nullptr))) return rc;
    n = (int)(s1 - s0);
  }
  if (steps) *steps = n;
  return EXA_OK;
}

int exa_lmesh_get_status(exa_lmesh* lm, int* h) {
  if (!lm || !h) return fail(EXA_ERR_ARG, "exa_lmesh_get_status: null argument");
  EXA_CUDA(cudaMemcpyAsync(h, lm->s, (size_t)lm->m->ncells * 4, cudaMemcpyDeviceToHost, lm->m->stream));
  EXA_CUDA(cudaStreamSynchronize(lm->m->stream));
  return EXA_OK;
}

int exa_lmesh_get_limiter(exa_lmesh* lm, double* lim, int* allocated) {
  if (!lm) return fail(EXA_ERR_ARG, "exa_lmesh_get_limiter: null mesh");
  const size_t n = lm->m->ncells;
  if (lim) EXA_CUDA(cudaMemcpyAsync(lim, lm->lim, n * lm->LS * 8, cudaMemcpyDeviceToHost, lm->m->stream));
  if (allocated) EXA_CUDA(cudaMemcpyAsync(allocated, lm->has_lim, n * 4, cudaMemcpyDeviceToHost, lm->m->stream));
  EXA_CUDA(cudaStreamSynchronize(lm->m->stream));
  return EXA_OK;
}

int exa_lmesh_set_priority(exa_lmesh* lm, int level) {
  if (!lm) return fail(EXA_ERR_ARG, "exa_lmesh_set_priority: null mesh");
  if (lm->graph) {  // captured on the old stream's priority
    cudaStreamSynchronize(lm->m->stream);
    cudaGraphExecDestroy(lm->graph);
    lm->graph = nullptr;
  }
  return exa_mesh_set_priority(lm->m, level);
}

int exa_lmesh_synchronize(exa_lmesh* lm) {
  if (!lm) return fail(EXA_ERR_ARG, "exa_lmesh_synchronize: null mesh");
  return exa_mesh_synchronize(lm->m);
}

int exa_lmesh_stream(exa_lmesh* lm, void** stream) {
  if (!lm) return fail(EXA_ERR_ARG, "exa_lmesh_stream: null mesh");
  return exa_mesh_stream(lm->m, stream);
}

}  // extern "C"

#include "batch.cuh"
