// C ABI of the FDTD engine: handle management, coefficient tables, TMA
// descriptors, launch selection and the step loops.  Declarations and the
// reference interface each entry point replaces: include/jaxphys_fdtd.h.
#include <cudaTypedefs.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/jaxphys_fdtd.h"
#include "fdtd2d_kernels.cuh"
#include "fdtd3d_adjoint.cuh"
#include "fdtd3d_kernels.cuh"
#include "learned_band.cuh"
#include "tb_registry.h"
#include "tma_registry.h"
#include "viz_kernels.cuh"

using namespace jxf;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------

static thread_local std::string g_last_error;

static int fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

#define CUDA_TRY(expr)                                                                   \
  do {                                                                                   \
    cudaError_t _e = (expr);                                                             \
    if (_e != cudaSuccess)                                                               \
      return fail(_e == cudaErrorMemoryAllocation ? JXF_ERR_OOM : JXF_ERR_CUDA,          \
                  "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(_e), __FILE__,      \
                  __LINE__);                                                             \
  } while (0)

#define TRY(expr)            \
  do {                       \
    int _rc = (expr);        \
    if (_rc != JXF_OK) return _rc; \
  } while (0)

namespace {

// physical constants, jaxphys src/neurosim/em/fdtd3d.py:36-38
constexpr double kC0 = 299792458.0;
constexpr double kPi = 3.14159265358979323846;
const double kMu0 = 4.0e-7 * kPi;
const double kEps0 = 1.0 / (kMu0 * kC0 * kC0);

// Make `dev` current for the duration of a call, restoring the caller's.
struct DeviceGuard {
  int prev = -1;
  bool ok = true;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) ok = (cudaSetDevice(dev) == cudaSuccess);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Fault injection for the failure-detection tests: JXF_FAULT_ALLOC_AFTER=n
// (read when a grid is created) lets the next n device allocations of that
// creation succeed and fails the one after with JXF_ERR_OOM.
thread_local long long g_alloc_budget = -1;

template <class T>
int dmalloc(T** p, size_t count, int64_t* tally) {
  *p = nullptr;
  if (count == 0) return JXF_OK;
  if (g_alloc_budget == 0) return fail(JXF_ERR_OOM, "device allocation refused (fault injection)");
  if (g_alloc_budget > 0) --g_alloc_budget;
  CUDA_TRY(cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T)));
  *tally += (int64_t)(count * sizeof(T));
  return JXF_OK;
}

template <class T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

template <class T>
int upload(T** p, const std::vector<T>& v, int64_t* tally) {
  dfree(*p);
  TRY(dmalloc(p, v.size(), tally));
  if (!v.empty()) CUDA_TRY(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return JXF_OK;
}

// Reference PML conductivity profile, fdtd3d.py:149-157 / fdtd.py:173-189:
// sigma_max*((n_pml-i)/n_pml)^3 at i and n-1-i, later writes winning.
std::vector<double> pml_sigma(int n, int n_pml, double dx) {
  std::vector<double> s(n, 0.0);
  if (n_pml <= 0) return s;
  const double sigma_max = 0.8 * 4.0 / (dx * 1.0);
  for (int i = 0; i < n_pml; ++i) {
    const double r = double(n_pml - i) / double(n_pml);
    const double val = sigma_max * r * r * r;
    if (i >= 0 && i < n) s[i] = val;
    if (n - 1 - i >= 0 && n - 1 - i < n) s[n - 1 - i] = val;
  }
  return s;
}

// Separable factor of exp(-sigma_avg dt/eps0) with sigma_avg = mean over `dims`
// axes (fdtd3d.py:221,363: dims=3; fdtd.py:242,344: dims=2).
std::vector<float> damping_table(int n, int n_pml, double dx, double dt, int dims) {
  std::vector<double> s = pml_sigma(n, n_pml, dx);
  std::vector<float> d(n);
  for (int i = 0; i < n; ++i) d[i] = (float)std::exp(-s[i] * dt / (kEps0 * dims));
  return d;
}

// CPML 1D tables (extension).  Depth rho in [0,1] from the nearest face,
// mirror-symmetric about (n-1)/2; sigma = sigma_max rho^m with
// sigma_max = -(m+1) ln R0 / (2 eta0 n_pml dx); kappa = 1 + (kappa_max-1) rho^m;
// alpha = alpha_max (1-rho); b = exp(-(sigma/kappa + alpha) dt/eps0);
// c = sigma (b-1) / (sigma kappa + kappa^2 alpha).
void cpml_tables(int n, int n_pml, double dx, double dt, double m, double r0, double kmax,
                 double amax, std::vector<float> out[TAB_COUNT]) {
  const double eta0 = std::sqrt(kMu0 / kEps0);
  const double smax = n_pml > 0 ? -(m + 1.0) * std::log(r0) / (2.0 * eta0 * n_pml * dx) : 0.0;
  for (int t = 0; t < TAB_COUNT; ++t) out[t].assign(n, 0.0f);
  for (int half = 0; half < 2; ++half) {
    for (int i = 0; i < n; ++i) {
      const double x = i + 0.5 * half;
      double rho = 0.0;
      if (n_pml > 0) {
        const double lo = (n_pml - x) / n_pml;
        const double hi = (x - (n - 1 - n_pml)) / n_pml;
        rho = std::min(1.0, std::max(0.0, std::max(lo, hi)));
      }
      const double pm = std::pow(rho, m);
      const double sigma = smax * pm;
      const double kappa = 1.0 + (kmax - 1.0) * pm;
      const double alpha = rho > 0.0 ? amax * (1.0 - rho) : 0.0;
      const double b = std::exp(-(sigma / kappa + alpha) * dt / kEps0);
      const double den = sigma * kappa + kappa * kappa * alpha;
      const double c = sigma > 0.0 ? sigma * (b - 1.0) / (den > 0.0 ? den : 1.0) : 0.0;
      const int base = half ? TAB_BH : TAB_BE;
      out[base + 0][i] = (float)b;
      out[base + 1][i] = (float)c;
      out[base + 2][i] = (float)(1.0 / kappa);
    }
  }
}

// ---------------------------------------------------------------------------
// TMA descriptors
// ---------------------------------------------------------------------------

PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

int get_encoder() {
  if (g_encode) return JXF_OK;
  void* fn = nullptr;
  cudaDriverEntryPointQueryResult q;
  CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
  if (q != cudaDriverEntryPointSuccess || fn == nullptr)
    return fail(JXF_ERR_CUDA, "cuTensorMapEncodeTiled not available from the driver");
  g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  return JXF_OK;
}

// Tiled map over a float32 (nx, ny, nz) array, box {bz, by, 1}.
int encode_map(CUtensorMap* m, const float* base, int nx, int ny, int nz, int bz, int by) {
  TRY(get_encoder());
  cuuint64_t dims[3] = {(cuuint64_t)nz, (cuuint64_t)ny, (cuuint64_t)nx};
  cuuint64_t strides[2] = {(cuuint64_t)nz * 4, (cuuint64_t)nz * ny * 4};
  cuuint32_t box[3] = {(cuuint32_t)bz, (cuuint32_t)by, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = g_encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(base), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(JXF_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return JXF_OK;
}

// ---------------------------------------------------------------------------
// TMA kernel registry
// ---------------------------------------------------------------------------

// autotune results: (nx, ny, nz, mode, cbarr) -> (cfg index, x_chunk, axis split,
// blocked cfg index or -1, blocked x_chunk)
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int, int>, std::tuple<int, int, int, int, int>> g_tune_cache;

}  // namespace

// ---------------------------------------------------------------------------
// 3D handle
// ---------------------------------------------------------------------------

// Device tables of a learned band attached to one grid or a batch: the grids'
// field pointers, the outer cells in single-face 128-cell tiles, the face of
// each tile and the correction buffer.
struct BandTables {
  jxf_band* band = nullptr;
  band::GridRef* d_grids = nullptr;    // fields of buffer set 0 of every grid
  band::GridRef* d_grids_b = nullptr;  // set 1 (TMA grids ping-pong; = set 0 otherwise)
  int2* d_cells = nullptr;
  int* d_tile_face = nullptr;
  float* d_delta = nullptr;
  int tiles = 0;
  int ctas = 0;
};

namespace {
int band_launch(const BandTables& t, cudaStream_t st, int set = 0);
void band_release(BandTables& t);
}  // namespace

struct jxf_grid3d {
  jxf_grid3d_desc d{};
  BandTables band;          // learned band (PEC, generic path), applied after each step
  int mode = MODE_ABSORB;   // kernel mode: ABSORB (also PEC with unit tables), PERIODIC, CPML
  // x-slab of a decomposed grid: local plane x is global plane x + gx0 of a
  // grid with gnx planes; planes [x_lo, x_hi) are owned, the two outer
  // planes are ghost copies of the neighbouring ranks' planes
  int gx0 = 0, gnx = 0, x_lo = 0, x_hi = 0;
  bool slab = false;
  bool kappa = false;       // CPML with kappa_max > 1 (1/kappa factors are not all 1)
  int path = JXF_PATH_GENERIC;
  double dt = 0, coef_h = 0, coef_e = 0;
  long long n = 0;
  int64_t bytes = 0;
  float* f[2][6] = {};
  float* cb = nullptr;
  float* damp[3] = {};
  float* tab[3][TAB_COUNT] = {};
  float* psi[2][PSI_COUNT] = {};
  int L[3] = {0, 0, 0}, P[3] = {-1, -1, -1};
  int cur = 0;
  long long step = 0;
  // sources (host copies kept to rebuild per-block lists)
  std::vector<long long> src_cell;
  std::vector<int> src_comp, src_wave;
  std::vector<float> src_amp;
  SrcCell* d_cells = nullptr;
  SrcTerm* d_terms = nullptr;
  int n_cells = 0;
  SrcEntry* d_entries = nullptr;
  int* d_blk_ptr = nullptr;
  int n_blocks_built = -1;
  int built_cfg = -1, built_chunk = -1;
  float* d_wave = nullptr;
  int n_waves = 0;
  long long wave_len = 0;
  // probes
  long long* d_probe_cell = nullptr;
  int* d_probe_comp = nullptr;
  int n_probes = 0;
  int* d_err = nullptr;
  int* d_count = nullptr;
  // CPML region split: blocks that touch a psi slab (shell) run the CPML
  // kernel, the others the plain kernel (compact block lists per launch shape)
  int* d_shell = nullptr;     // shell blocks touching slabs of several axes
  int* d_shell_ax[3] = {};    // shell blocks touching the slab of one axis (x, y, z)
  int* d_inner = nullptr;
  int n_shell = 0, n_inner = 0;
  int n_shell_ax[3] = {0, 0, 0};
  int axis_split = 0;         // run single-axis shell blocks on the specialised kernels
  int split_axes = -1;        // axis_split the current block lists were built for
  int split_cfg = -1, split_chunk = -1;
  bool use_pdl = true;  // programmatic dependent launch between step kernels
  // adjoint (sqrt(T) checkpointing): checkpoints of the full state every
  // adj_k steps, one segment of per-step (H, psiE) snapshots, adjoint state
  int adj_n = 0, adj_k = 0, adj_nseg = 0;
  size_t adj_state = 0, adj_segstate = 0;  // floats per checkpoint / per snapshot
  float* adj_ck = nullptr;
  float* adj_sg = nullptr;
  float* adj_l = nullptr;   // lE(3n) lH(3n) lpsi(psi) db(6n) dh(6n)
  double* adj_g = nullptr;  // dJ/dcb
  size_t adj_ck_cap = 0, adj_sg_cap = 0, adj_l_cap = 0, adj_g_cap = 0;
  // TMA selection
  int cfg = -1, x_chunk = 0;
  bool maps_ok = false;
  int maps_cfg = -1;  // config whose box shapes the maps were encoded with
  Maps3D maps[2];     // input set 0 / 1
  // two-level temporally blocked launches (tb_registry.h): tb = registry
  // index, or -1 for one step per launch
  int tb = -1, tb_chunk = 0;
  bool maps_tb_ok = false;
  int maps_tb_cfg = -1;
  MapsTB maps_tb[2];
  std::vector<long long> probe_cell_h;  // host copies for the per-block probe lists
  std::vector<int> probe_comp_h;
  TbSrc* d_tb_src = nullptr;
  int* d_tb_src_ptr = nullptr;
  TbProbe* d_tb_probe = nullptr;
  int* d_tb_probe_ptr = nullptr;
  int tb_built_cfg = -1, tb_built_chunk = -1;
  int* d_tb_shell = nullptr;
  int* d_tb_shell_ax[6] = {};  // one axis (x, y, z), two axes (xy, xz, yz)
  int* d_tb_inner = nullptr;
  int n_tb_shell = 0, n_tb_inner = 0;
  int n_tb_shell_ax[6] = {0, 0, 0, 0, 0, 0};
  int tb_split_cfg = -1, tb_split_chunk = -1, tb_split_axes = -1;
};

namespace {

int cells_ok(const jxf_grid3d* g, long long cell) { return cell >= 0 && cell < g->n; }

int build_generic_sources(jxf_grid3d* g) {
  // group by (cell, comp) in order of first appearance; terms in list order
  std::map<std::pair<long long, int>, std::vector<int>> groups;
  std::vector<std::pair<long long, int>> order;
  for (size_t i = 0; i < g->src_cell.size(); ++i) {
    auto key = std::make_pair(g->src_cell[i], g->src_comp[i]);
    auto it = groups.find(key);
    if (it == groups.end()) {
      order.push_back(key);
      groups[key] = {(int)i};
    } else {
      it->second.push_back((int)i);
    }
  }
  std::vector<SrcCell> cells;
  std::vector<SrcTerm> terms;
  for (auto& key : order) {
    SrcCell c{};
    c.cell = key.first;
    c.comp = key.second;
    c.first = (int)terms.size();
    for (int i : groups[key]) terms.push_back(SrcTerm{g->src_amp[i], g->src_wave[i]});
    c.count = (int)terms.size() - c.first;
    cells.push_back(c);
  }
  g->n_cells = (int)cells.size();
  TRY(upload(&g->d_cells, cells, &g->bytes));
  TRY(upload(&g->d_terms, terms, &g->bytes));
  return JXF_OK;
}

// Local planes [beg, end) that the one-step TMA pass marches over, in chunks
// of x_chunk from beg (the kernel derives the same range from gx0 and x_hi):
// every plane of a whole grid; the owned planes of an x-slab and its left
// ghost plane (H recomputed there), unless that ghost lies outside the grid.
void march_range(const jxf_grid3d* g, int& beg, int& end) {
  beg = g->gx0 < 0 ? 1 : 0;
  end = g->x_hi;
}
int march_chunks(const jxf_grid3d* g, int chunk) {
  int beg, end;
  march_range(g, beg, end);
  return (end - beg + chunk - 1) / chunk;
}

// Per-block source lists for the TMA kernel: CSR over blocks, entries sorted
// by plane, list order kept inside a plane (stable sort).  Sources on the
// ghost planes of an x-slab belong to the neighbour and are left out.
int build_tma_sources(jxf_grid3d* g) {
  const TmaConfig& c = tma_configs()[g->cfg];
  const int ny = g->d.ny, nz = g->d.nz;
  const int ntz = (nz + c.tz - 1) / c.tz, nty = (ny + c.ty - 1) / c.ty;
  int xbeg, xend;
  march_range(g, xbeg, xend);
  const int nch = march_chunks(g, g->x_chunk);
  const int nblk = ntz * nty * nch;
  std::vector<std::pair<int, int>> keyed;  // (block, source index)
  for (size_t i = 0; i < g->src_cell.size(); ++i) {
    const long long cell = g->src_cell[i];
    const int z = (int)(cell % nz);
    const int y = (int)((cell / nz) % ny);
    const int x = (int)(cell / ((long long)nz * ny));
    if (x < g->x_lo || x >= g->x_hi) continue;
    const int b = (((x - xbeg) / g->x_chunk) * nty + y / c.ty) * ntz + z / c.tz;
    keyed.push_back({b, (int)i});
  }
  std::stable_sort(keyed.begin(), keyed.end(), [&](const auto& u, const auto& v) {
    if (u.first != v.first) return u.first < v.first;
    const long long xu = g->src_cell[u.second] / ((long long)nz * ny);
    const long long xv = g->src_cell[v.second] / ((long long)nz * ny);
    return xu < xv;
  });
  std::vector<int> ptr(nblk + 1, 0);
  std::vector<SrcEntry> ents;
  for (auto& kv : keyed) {
    const int i = kv.second;
    const long long cell = g->src_cell[i];
    const int z = (int)(cell % nz);
    const int y = (int)((cell / nz) % ny);
    const int x = (int)(cell / ((long long)nz * ny));
    SrcEntry e{};
    e.x = x;
    e.off = (y % c.ty) * c.tz + (z % c.tz);
    e.comp = g->src_comp[i];
    e.wave = g->src_wave[i];
    e.amp = g->src_amp[i];
    ents.push_back(e);
    ptr[kv.first + 1]++;
  }
  for (int b = 0; b < nblk; ++b) ptr[b + 1] += ptr[b];
  TRY(upload(&g->d_entries, ents, &g->bytes));
  TRY(upload(&g->d_blk_ptr, ptr, &g->bytes));
  g->built_cfg = g->cfg;
  g->built_chunk = g->x_chunk;
  return JXF_OK;
}

int encode_maps(jxf_grid3d* g) {
  const TmaConfig& c = tma_configs()[g->cfg];
  const int nx = g->d.nx, ny = g->d.ny, nz = g->d.nz;
  for (int s = 0; s < 2; ++s) {
    for (int k = 0; k < 3; ++k) {
      TRY(encode_map(&g->maps[s].e[k], g->f[s][k], nx, ny, nz, c.tz + 8, c.ty + 2));
      TRY(encode_map(&g->maps[s].h[k], g->f[s][3 + k], nx, ny, nz, c.tz + 4, c.ty + 1));
    }
    if (g->cb) {
      TRY(encode_map(&g->maps[s].cb, g->cb, nx, ny, nz, c.tz, c.ty));
    } else {
      g->maps[s].cb = g->maps[s].e[0];  // unused
    }
  }
  g->maps_ok = true;
  g->maps_cfg = g->cfg;
  return JXF_OK;
}

// Bound on every device-side wait: 2 s, or JXF_WAIT_LIMIT_MS.
unsigned long long wait_limit_ns() {
  static unsigned long long v = [] {
    const char* e = std::getenv("JXF_WAIT_LIMIT_MS");
    long long ms = e ? std::atoll(e) : 2000;
    if (ms < 1) ms = 1;
    return (unsigned long long)ms * 1000000ull;
  }();
  return v;
}

// Fault injection for the failure-detection tests, read at every step call:
// JXF_FAULT_DROP_STAGE=l makes every block of the TMA step kernels skip the
// copy of its l-th staged plane (its bounded waits then run out and the step
// reports JXF_ERR_TIMEOUT through jxf_grid3d_check_error).
int fault_drop_stage() {
  const char* e = std::getenv("JXF_FAULT_DROP_STAGE");
  if (!e || !*e) return -1;
  const int v = std::atoi(e);
  return v >= 0 ? v : -1;
}

Step3D base_params(jxf_grid3d* g) {
  Step3D p{};
  p.drop_stage = fault_drop_stage();
  p.nx = g->d.nx;
  p.ny = g->d.ny;
  p.nz = g->d.nz;
  p.a = (float)g->coef_h;
  p.cb_const = (float)g->coef_e;
  p.cb = g->cb;
  for (int k = 0; k < 3; ++k) p.damp[k] = g->damp[k];
  for (int ax = 0; ax < 3; ++ax) {
    for (int t = 0; t < TAB_COUNT; ++t) p.pml.tab[ax][t] = g->tab[ax][t];
    p.pml.L[ax] = g->L[ax];
    p.pml.P[ax] = g->P[ax];
  }
  p.wave = g->d_wave;
  p.wave_len = g->wave_len;
  p.n_probes = g->n_probes;
  p.probe_cell = g->d_probe_cell;
  p.probe_comp = g->d_probe_comp;
  p.err = g->d_err;
  p.wait_ns = wait_limit_ns();
  p.gx0 = g->gx0;
  p.gnx = g->gnx;
  p.x_lo = g->x_lo;
  p.x_hi = g->x_hi;
  p.div_nz = make_fastdiv((uint32_t)g->d.nz);
  p.div_ny = make_fastdiv((uint32_t)g->d.ny);
  p.idx32 = ((long long)g->d.nx * g->d.ny * g->d.nz) < (1ll << 32) ? 1 : 0;
  return p;
}

void set_io(jxf_grid3d* g, Step3D& p, int in_set, int out_set) {
  for (int k = 0; k < 6; ++k) {
    p.in[k] = g->f[in_set][k];
    p.out[k] = g->f[out_set][k];
  }
  for (int k = 0; k < PSI_COUNT; ++k) {
    p.pml.in[k] = g->psi[in_set][k];
    p.pml.out[k] = g->psi[out_set][k];
  }
}

int launch_tma(jxf_grid3d* g, int cfg, int chunk, Step3D& p, int in_set, cudaStream_t st,
               int list_count, bool plain = false, int axis = -1) {
  // The boxes of the tensor maps must be the ones this config's kernel expects
  // (the mbarrier transaction count is derived from them).
  if (!g->maps_ok || g->maps_cfg != cfg)
    return fail(JXF_ERR_INVALID, "tensor maps encoded for config %d, launching config %d",
                g->maps_cfg, cfg);
  const TmaConfig& c = tma_configs()[cfg];
  const bool cpml = g->mode == MODE_CPML && !plain;
  const int mi = cpml ? 1 : 0;
  const int ki = cpml ? (g->kappa ? 2 : 1) : 0;
  TmaKernel k = c.k[ki][g->cb ? 1 : 0];
  size_t smem = c.smem[mi];
  if (cpml && axis >= 0) {  // single-axis shell blocks (kappa = 1 only)
    k = c.kax[axis][g->cb ? 1 : 0];
    smem = c.smem_ax[axis];
  }
  {
    // the shared-memory opt-in is set once per kernel and device (a driver
    // call per launch would make small steps host bound)
    static std::mutex mu;
    static std::map<std::pair<TmaKernel, int>, size_t> done;
    std::lock_guard<std::mutex> lk(mu);
    size_t& have = done[{k, g->d.device}];
    if (have < smem) {
      CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      // the carveout is a hint the driver may undercut (down to one block per
      // SM for the large-tile shapes): ask for the largest shared split
      CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    cudaSharedmemCarveoutMaxShared));
      have = smem;
    }
  }
  p.x_chunk = chunk;
  p.ntiles_z = (g->d.nz + c.tz - 1) / c.tz;
  p.ntiles_y = (g->d.ny + c.ty - 1) / c.ty;
  dim3 grid(p.ntiles_z, p.ntiles_y, march_chunks(g, chunk));
  if (list_count >= 0) grid = dim3(list_count, 1, 1);
  cudaLaunchConfig_t lc{};
  lc.gridDim = grid;
  lc.blockDim = dim3(c.threads, 1, 1);
  lc.dynamicSmemBytes = smem;
  lc.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = g->use_pdl ? 1 : 0;
  lc.attrs = attr;
  lc.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&lc, k, p, g->maps[in_set]);
  if (e != cudaSuccess && g->use_pdl) {
    // stream without programmatic serialization support: launch in order
    (void)cudaGetLastError();
    g->use_pdl = false;
    p.pdl = 0;
    lc.numAttrs = 0;
    e = cudaLaunchKernelEx(&lc, k, p, g->maps[in_set]);
  }
  if (e != cudaSuccess)
    return fail(JXF_ERR_CUDA, "step kernel launch failed: %s", cudaGetErrorString(e));
  return JXF_OK;
}

// A coordinate range [lo, hi] along an axis of length n avoids the slab
// storage of half width P (P < 0: the whole axis is stored).
bool range_clear(int lo, int hi, int n, int P) {
  if (P < 0) return false;
  lo = std::max(lo, 0);
  hi = std::min(hi, n - 1);
  return lo >= P && hi < n - P;
}

// JXF_SLAB_FIRST=0 keeps the row-major cell order in every CPML block.
bool slab_first_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("JXF_SLAB_FIRST");
    return !(e && e[0] == '0');
  }();
  return on;
}

// JXF_BLOCK_ORDER=0 launches the CPML shell blocks in grid order instead of
// heaviest first.
bool heavy_first_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("JXF_BLOCK_ORDER");
    return !(e && e[0] == '0');
  }();
  return on;
}

bool in_slab(int i, int n, int P) { return P < 0 || i < P || i >= n - P; }

// Work of a CPML shell block in warp-planes: a warp holding a slab cell runs
// the CPML update (counted 2), the others the plain one (1); every warp of a
// plane inside the x slab runs CPML; the warm-up plane counts half.  All the
// blocks of a small grid are resident at once, so the step lasts as long as
// the most loaded SM: launching the blocks heaviest first spreads the heavy
// ones over the SMs (the hardware hands out blocks in launch order).
// Warps of a tile that run the CPML update on planes outside the x slab.
int tile_cpml_warps(const jxf_grid3d* g, const TmaConfig& c, int z0, int y0, bool slab_first) {
  const int ny = g->d.ny, nz = g->d.nz;
  const int threads = c.threads, warps = (threads + 31) / 32;
  std::vector<char> warp_cpml(warps, 0);
  int n_cpml = 0;
  for (int t = 0; t < threads; ++t) {
    const int tx = t % c.tz, tyt = t / c.tz;
    bool any = false;
    for (int r = 0; r < c.ry; ++r) {
      const int y = y0 + tyt + r * (c.ty / c.ry), z = z0 + tx;
      if (y < ny && z < nz && (in_slab(y, ny, g->P[1]) || in_slab(z, nz, g->P[2]))) any = true;
    }
    if (any) {
      ++n_cpml;
      warp_cpml[t / 32] = 1;
    }
  }
  return slab_first ? (n_cpml + 31) / 32 : (int)std::count(warp_cpml.begin(), warp_cpml.end(), 1);
}

double shell_block_cost(const jxf_grid3d* g, const TmaConfig& c, int cw, int xb, int xe) {
  const int warps = (c.threads + 31) / 32;
  double cost = 0.0;
  for (int x = std::max(xb - 1, 0); x < xe; ++x) {
    const bool xin = in_slab(x + g->gx0, g->gnx, g->P[0]);
    const double plane = xin ? 2.0 * warps : 2.0 * cw + (warps - cw);
    cost += x < xb ? 0.5 * plane : plane;
  }
  return cost;
}

// Block lists of a CPML grid at one launch shape: shell blocks that touch the
// slabs of several axes, of one axis (x, y, z), and interior blocks, each as
// (tile_z, tile_y, chunk word) triples with a work estimate, heaviest first.
struct SplitLists {
  std::vector<int> list[5];     // [0 shell, 1..3 single-axis x/y/z, 4 interior]
  std::vector<double> cost[5];  // per block
};

void compute_split(const jxf_grid3d* g, int cfg, int chunk, bool axis_split, SplitLists& out) {
  const TmaConfig& c = tma_configs()[cfg];
  const int ny = g->d.ny, nz = g->d.nz;
  const int ntz = (nz + c.tz - 1) / c.tz, nty = (ny + c.ty - 1) / c.ty;
  int xbeg, xend;
  march_range(g, xbeg, xend);
  const int nch = march_chunks(g, chunk);
  struct Blk {
    double cost;
    int tz, ty, word;
  };
  std::vector<Blk> parts[5];
  std::vector<int> tile_cw((size_t)ntz * nty, -1);  // filled on first use
  const int warps = (c.threads + 31) / 32;
  for (int ch = 0; ch < nch; ++ch)
    for (int ty = 0; ty < nty; ++ty)
      for (int tz = 0; tz < ntz; ++tz) {
        const int z0 = tz * c.tz, y0 = ty * c.ty, xb = xbeg + ch * chunk;
        const int xe = std::min(xb + chunk, xend);
        // cells of the tile, its halo row / column, and the warm-up plane
        // (x in global planes)
        const bool cz = range_clear(z0 - 1, z0 + c.tz - 1, nz, g->P[2]);
        const bool cy = range_clear(y0 - 1, y0 + c.ty - 1, ny, g->P[1]);
        const bool cx = range_clear(xb - 1 + g->gx0, xe - 1 + g->gx0, g->gnx, g->P[0]);
        const int touched = (cx ? 0 : 1) + (cy ? 0 : 1) + (cz ? 0 : 1);
        if (touched == 0) {
          parts[4].push_back({(double)(xe - std::max(xb - 1, 0)) * warps, tz, ty, ch});
          continue;
        }
        int pi = 0;
        if (touched == 1 && !g->kappa && axis_split) pi = 1 + (!cx ? 0 : (!cy ? 1 : 2));
        // blocks holding z-slab cells order them first (one row per thread)
        const bool slab_first = !cz && c.ry == 1 && slab_first_enabled();
        int& cw = tile_cw[(size_t)ty * ntz + tz];
        if (cw < 0) cw = tile_cpml_warps(g, c, z0, y0, slab_first);
        parts[pi].push_back({shell_block_cost(g, c, cw, xb, xe), tz, ty,
                             ch | (slab_first ? BLK_SLAB_FIRST : 0)});
      }
  for (int k = 0; k < 5; ++k) {
    if (k < 4 && heavy_first_enabled())
      std::stable_sort(parts[k].begin(), parts[k].end(),
                       [](const Blk& u, const Blk& v) { return u.cost > v.cost; });
    out.list[k].clear();
    out.cost[k].clear();
    for (const Blk& b : parts[k]) {
      out.list[k].push_back(b.tz);
      out.list[k].push_back(b.ty);
      out.list[k].push_back(b.word);
      out.cost[k].push_back(b.cost);
    }
  }
}

int build_split(jxf_grid3d* g, int cfg, int chunk) {
  if (g->split_cfg == cfg && g->split_chunk == chunk && g->split_axes == g->axis_split)
    return JXF_OK;
  SplitLists sl;
  compute_split(g, cfg, chunk, g->axis_split != 0, sl);
  TRY(upload(&g->d_shell, sl.list[0], &g->bytes));
  TRY(upload(&g->d_inner, sl.list[4], &g->bytes));
  for (int a = 0; a < 3; ++a) {
    TRY(upload(&g->d_shell_ax[a], sl.list[1 + a], &g->bytes));
    g->n_shell_ax[a] = (int)sl.list[1 + a].size() / 3;
  }
  g->n_shell = (int)sl.list[0].size() / 3;
  g->n_inner = (int)sl.list[4].size() / 3;
  g->split_cfg = cfg;
  g->split_chunk = chunk;
  g->split_axes = g->axis_split;
  return JXF_OK;
}

// One leapfrog step on the TMA path.  CPML grids: the CPML kernel over the
// shell blocks that touch the slabs of several axes, the single-axis CPML
// variants over the blocks that touch one axis's slab, then the plain kernel
// over the interior blocks (disjoint outputs, all read the same input set).
// Programmatic dependent launch chains them: the first launch waits for the
// previous step, each later one starts beside its predecessor and waits for
// it before exiting, so the last one's completion covers the whole step.
int launch_step(jxf_grid3d* g, int cfg, int chunk, Step3D& p, int in_set, cudaStream_t st) {
  p.pdl = g->use_pdl ? (PDL_WAIT_START | PDL_TRIGGER) : 0;
  if (g->mode != MODE_CPML) {
    p.blk_list = nullptr;
    return launch_tma(g, cfg, chunk, p, in_set, st, -1);
  }
  TRY(build_split(g, cfg, chunk));
  struct Part {
    const int* list;
    int n;
    bool plain;
    int axis;
  };
  const Part parts[5] = {{g->d_shell, g->n_shell, false, -1},
                         {g->d_shell_ax[0], g->n_shell_ax[0], false, 0},
                         {g->d_shell_ax[1], g->n_shell_ax[1], false, 1},
                         {g->d_shell_ax[2], g->n_shell_ax[2], false, 2},
                         {g->d_inner, g->n_inner, true, -1}};
  bool first = true;
  for (const Part& part : parts) {
    if (part.n <= 0) continue;
    Step3D q = p;
    q.blk_list = part.list;
    if (!first) {
      q.probe_out = nullptr;
      if (g->use_pdl) q.pdl = PDL_TRIGGER | PDL_WAIT_END;
    }
    TRY(launch_tma(g, cfg, chunk, q, in_set, st, part.n, part.plain, part.axis));
    first = false;
  }
  return JXF_OK;
}

// ---------------------------------------------------------------------------
// two-level temporally blocked launches (fdtd3d_tb.cuh)
// ---------------------------------------------------------------------------

int tb_ntiles_z(const jxf_grid3d* g) { return (g->d.nz + TB_TZ - 1) / TB_TZ; }
int tb_ntiles_y(const jxf_grid3d* g, const TbConfig& c) { return (g->d.ny + c.ty - 1) / c.ty; }

int encode_maps_tb(jxf_grid3d* g) {
  const TbConfig& c = tb_configs()[g->tb];
  const int nx = g->d.nx, ny = g->d.ny, nz = g->d.nz;
  for (int s = 0; s < 2; ++s) {
    for (int k = 0; k < 3; ++k) {
      TRY(encode_map(&g->maps_tb[s].e[k], g->f[s][k], nx, ny, nz, TB_BW, c.nr + 1));
      TRY(encode_map(&g->maps_tb[s].h[k], g->f[s][3 + k], nx, ny, nz, TB_BW, c.nr));
    }
    if (g->cb) {
      TRY(encode_map(&g->maps_tb[s].cb, g->cb, nx, ny, nz, TB_BW, c.nr));
    } else {
      g->maps_tb[s].cb = g->maps_tb[s].e[0];  // unused
    }
  }
  g->maps_tb_ok = true;
  g->maps_tb_cfg = g->tb;
  return JXF_OK;
}

// Per-block source and probe lists of the blocked kernel (CSR over blocks in
// grid order, entries sorted by plane, list order kept inside a plane).  A
// source enters every block whose region (tile plus the two-cell halo) and
// level-1 planes hold its cell: level 1 (step n) adds it to every region
// cell; level 2 (step n+1) only on the owner's tile.  A probe enters its
// owner block only.
int build_tb_lists(jxf_grid3d* g) {
  const TbConfig& c = tb_configs()[g->tb];
  const int nx = g->d.nx, ny = g->d.ny, nz = g->d.nz, chunk = g->tb_chunk;
  const int ntz = tb_ntiles_z(g), nty = tb_ntiles_y(g, c), nch = (nx + chunk - 1) / chunk;
  const int nblk = ntz * nty * nch;
  struct Keyed {
    int blk, x, order;
    TbSrc e;
  };
  std::vector<Keyed> ks;
  for (size_t i = 0; i < g->src_cell.size(); ++i) {
    const long long cell = g->src_cell[i];
    const int z = (int)(cell % nz);
    const int y = (int)((cell / nz) % ny);
    const int x = (int)(cell / ((long long)nz * ny));
    for (int ch = std::max(0, x / chunk - 1); ch <= std::min(nch - 1, (x + 2) / chunk); ++ch) {
      const int xb = ch * chunk, xe = std::min(xb + chunk, nx);
      const int qs = std::max(xb - 2, 0), q1 = std::min(xe, nx - 1);
      if (x < qs || x > q1) continue;
      for (int ty = std::max(0, (y + 2) / c.ty - 2); ty <= std::min(nty - 1, (y + 2) / c.ty + 1);
           ++ty) {
        const int y0 = ty * c.ty;
        if (y < y0 - 2 || y > y0 - 2 + c.nr - 1) continue;
        for (int tz = std::max(0, (z + 2) / TB_TZ - 2);
             tz <= std::min(ntz - 1, (z + 2) / TB_TZ + 1); ++tz) {
          const int z0 = tz * TB_TZ;
          if (z < z0 - 2 || z > z0 + 29) continue;
          const bool tile = y >= y0 && y < y0 + c.ty && z >= z0 && z < z0 + TB_TZ;
          TbSrc e{};
          e.x = x;
          e.off = (y - (y0 - 2)) * 32 + (z - (z0 - 2));
          e.comp = g->src_comp[i];
          e.wave = g->src_wave[i];
          e.amp = g->src_amp[i];
          e.lv = 1 | ((tile && x >= xb && x < xe) ? 2 : 0);
          ks.push_back({(ch * nty + ty) * ntz + tz, x, (int)i, e});
        }
      }
    }
  }
  std::stable_sort(ks.begin(), ks.end(), [](const Keyed& u, const Keyed& v) {
    if (u.blk != v.blk) return u.blk < v.blk;
    return u.x < v.x;
  });
  std::vector<int> ptr(nblk + 1, 0);
  std::vector<TbSrc> ents;
  ents.reserve(ks.size());
  for (const Keyed& k : ks) {
    ents.push_back(k.e);
    ptr[k.blk + 1]++;
  }
  for (int b = 0; b < nblk; ++b) ptr[b + 1] += ptr[b];
  TRY(upload(&g->d_tb_src, ents, &g->bytes));
  TRY(upload(&g->d_tb_src_ptr, ptr, &g->bytes));

  struct KeyedP {
    int blk, x;
    TbProbe e;
  };
  std::vector<KeyedP> kp;
  for (size_t j = 0; j < g->probe_cell_h.size(); ++j) {
    const long long cell = g->probe_cell_h[j];
    const int z = (int)(cell % nz);
    const int y = (int)((cell / nz) % ny);
    const int x = (int)(cell / ((long long)nz * ny));
    const int tz = z / TB_TZ, ty = y / c.ty, ch = x / chunk;
    TbProbe e{};
    e.x = x;
    e.off = (y - (ty * c.ty - 2)) * 32 + (z - (tz * TB_TZ - 2));
    e.comp = g->probe_comp_h[j];
    e.slot = (int)j;
    kp.push_back({(ch * nty + ty) * ntz + tz, x, e});
  }
  std::stable_sort(kp.begin(), kp.end(), [](const KeyedP& u, const KeyedP& v) {
    if (u.blk != v.blk) return u.blk < v.blk;
    return u.x < v.x;
  });
  std::vector<int> pptr(nblk + 1, 0);
  std::vector<TbProbe> pents;
  for (const KeyedP& k : kp) {
    pents.push_back(k.e);
    pptr[k.blk + 1]++;
  }
  for (int b = 0; b < nblk; ++b) pptr[b + 1] += pptr[b];
  TRY(upload(&g->d_tb_probe, pents, &g->bytes));
  TRY(upload(&g->d_tb_probe_ptr, pptr, &g->bytes));
  g->tb_built_cfg = g->tb;
  g->tb_built_chunk = chunk;
  return JXF_OK;
}

// CPML grids: blocks whose region (tile, two-cell halo, level-1 planes)
// touches the psi slabs of several axes, of one axis, or none.
int build_tb_split(jxf_grid3d* g, int cfg, int chunk) {
  if (g->tb_split_cfg == cfg && g->tb_split_chunk == chunk && g->tb_split_axes == g->axis_split)
    return JXF_OK;
  const TbConfig& c = tb_configs()[cfg];
  const int nx = g->d.nx, ny = g->d.ny, nz = g->d.nz;
  const int ntz = tb_ntiles_z(g), nty = tb_ntiles_y(g, c);
  const int nch = (nx + chunk - 1) / chunk;
  struct Blk {
    int cost, tz, ty, ch;
  };
  std::vector<Blk> shell_b, axl_b[6];
  std::vector<int> inner;
  const bool axis_split = g->axis_split != 0;
  for (int ch = 0; ch < nch; ++ch)
    for (int ty = 0; ty < nty; ++ty)
      for (int tz = 0; tz < ntz; ++tz) {
        const int z0 = tz * TB_TZ, y0 = ty * c.ty, xb = ch * chunk;
        const int xe = std::min(xb + chunk, nx);
        const bool cz = range_clear(z0 - 2, z0 + 29, nz, g->P[2]);
        const bool cy = range_clear(y0 - 2, y0 + c.nr - 3, ny, g->P[1]);
        const bool cx = range_clear(std::max(xb - 2, 0), std::min(xe, nx - 1), nx, g->P[0]);
        const int touched = (cx ? 0 : 1) + (cy ? 0 : 1) + (cz ? 0 : 1);
        if (touched == 0) {
          inner.push_back(tz);
          inner.push_back(ty);
          inner.push_back(ch);
          continue;
        }
        int xs = 0;  // level-1 planes inside the x slab
        for (int x = std::max(xb - 2, 0); x <= std::min(xe, nx - 1); ++x)
          xs += in_slab(x, nx, g->P[0]) ? 1 : 0;
        std::vector<Blk>* v = &shell_b;
        if (touched == 1 && !g->kappa && axis_split) v = &axl_b[!cx ? 0 : (!cy ? 1 : 2)];
        // two axes: xy, xz, yz
        if (touched == 2 && !g->kappa && axis_split) v = &axl_b[cz ? 3 : (cy ? 4 : 5)];
        v->push_back({touched * 4096 + xs, tz, ty, ch});
      }
  auto flatten = [&](std::vector<Blk>& in, std::vector<int>& out) {
    if (heavy_first_enabled())
      std::stable_sort(in.begin(), in.end(),
                       [](const Blk& u, const Blk& v) { return u.cost > v.cost; });
    for (const Blk& b : in) {
      out.push_back(b.tz);
      out.push_back(b.ty);
      out.push_back(b.ch);
    }
  };
  std::vector<int> shell, axl[6];
  flatten(shell_b, shell);
  for (int a = 0; a < 6; ++a) flatten(axl_b[a], axl[a]);
  TRY(upload(&g->d_tb_shell, shell, &g->bytes));
  TRY(upload(&g->d_tb_inner, inner, &g->bytes));
  for (int a = 0; a < 6; ++a) {
    TRY(upload(&g->d_tb_shell_ax[a], axl[a], &g->bytes));
    g->n_tb_shell_ax[a] = (int)axl[a].size() / 3;
  }
  g->n_tb_shell = (int)shell.size() / 3;
  g->n_tb_inner = (int)inner.size() / 3;
  g->tb_split_cfg = cfg;
  g->tb_split_chunk = chunk;
  g->tb_split_axes = g->axis_split;
  return JXF_OK;
}

int launch_tb(jxf_grid3d* g, int cfg, int chunk, Step3D& p, const TbExtra& ex, int in_set,
              cudaStream_t st, int list_count, bool plain = false, int axis = -1) {
  if (!g->maps_tb_ok || g->maps_tb_cfg != cfg)
    return fail(JXF_ERR_INVALID, "blocked tensor maps encoded for config %d, launching %d",
                g->maps_tb_cfg, cfg);
  const TbConfig& c = tb_configs()[cfg];
  const bool cpml = g->mode == MODE_CPML && !plain;
  const int ki = cpml ? (g->kappa ? 2 : 1) : 0;
  TbKernel k = c.k[ki][g->cb ? 1 : 0];
  size_t smem = c.smem[cpml ? 1 : 0];
  if (cpml && axis >= 0 && axis < 3) {
    k = c.kax[axis][g->cb ? 1 : 0];
    smem = c.smem_ax[axis];
  } else if (cpml && axis >= 3) {
    k = c.kax2[axis - 3][g->cb ? 1 : 0];
    smem = c.smem_ax2[axis - 3];
  }
  {
    static std::mutex mu;
    static std::map<std::pair<TbKernel, int>, size_t> done;
    std::lock_guard<std::mutex> lk(mu);
    size_t& have = done[{k, g->d.device}];
    if (have < smem) {
      CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                    cudaSharedmemCarveoutMaxShared));
      have = smem;
    }
  }
  p.x_chunk = chunk;
  p.ntiles_z = tb_ntiles_z(g);
  p.ntiles_y = tb_ntiles_y(g, c);
  dim3 grid(p.ntiles_z, p.ntiles_y, (g->d.nx + chunk - 1) / chunk);
  if (list_count >= 0) grid = dim3(list_count, 1, 1);
  cudaLaunchConfig_t lc{};
  lc.gridDim = grid;
  lc.blockDim = dim3(c.threads, 1, 1);
  lc.dynamicSmemBytes = smem;
  lc.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = g->use_pdl ? 1 : 0;
  lc.attrs = attr;
  lc.numAttrs = 1;
  cudaError_t e = cudaLaunchKernelEx(&lc, k, p, g->maps_tb[in_set], ex);
  if (e != cudaSuccess && g->use_pdl) {
    (void)cudaGetLastError();
    g->use_pdl = false;
    p.pdl = 0;
    lc.numAttrs = 0;
    e = cudaLaunchKernelEx(&lc, k, p, g->maps_tb[in_set], ex);
  }
  if (e != cudaSuccess)
    return fail(JXF_ERR_CUDA, "blocked step kernel launch failed: %s", cudaGetErrorString(e));
  return JXF_OK;
}

// Two leapfrog steps in one pass (per part for CPML grids, chained by
// programmatic dependent launch as in launch_step).
int launch_tb_step(jxf_grid3d* g, int cfg, int chunk, Step3D& p, const TbExtra& ex, int in_set,
                   cudaStream_t st) {
  p.pdl = g->use_pdl ? (PDL_WAIT_START | PDL_TRIGGER) : 0;
  if (g->mode != MODE_CPML) {
    p.blk_list = nullptr;
    return launch_tb(g, cfg, chunk, p, ex, in_set, st, -1);
  }
  TRY(build_tb_split(g, cfg, chunk));
  struct Part {
    const int* list;
    int n;
    bool plain;
    int axis;
  };
  const Part parts[8] = {{g->d_tb_shell, g->n_tb_shell, false, -1},
                         {g->d_tb_shell_ax[3], g->n_tb_shell_ax[3], false, 3},
                         {g->d_tb_shell_ax[4], g->n_tb_shell_ax[4], false, 4},
                         {g->d_tb_shell_ax[5], g->n_tb_shell_ax[5], false, 5},
                         {g->d_tb_shell_ax[0], g->n_tb_shell_ax[0], false, 0},
                         {g->d_tb_shell_ax[1], g->n_tb_shell_ax[1], false, 1},
                         {g->d_tb_shell_ax[2], g->n_tb_shell_ax[2], false, 2},
                         {g->d_tb_inner, g->n_tb_inner, true, -1}};
  bool first = true;
  for (const Part& part : parts) {
    if (part.n <= 0) continue;
    Step3D q = p;
    q.blk_list = part.list;
    if (!first) {
      q.probe_out = nullptr;
      if (g->use_pdl) q.pdl = PDL_TRIGGER | PDL_WAIT_END;
    }
    TRY(launch_tb(g, cfg, chunk, q, ex, in_set, st, part.n, part.plain, part.axis));
    first = false;
  }
  return JXF_OK;
}

TbExtra tb_extra(const jxf_grid3d* g, float* probe_mid) {
  TbExtra ex{};
  ex.src_ptr = g->src_cell.empty() ? nullptr : g->d_tb_src_ptr;
  ex.src = g->d_tb_src;
  ex.probe_ptr = g->n_probes > 0 ? g->d_tb_probe_ptr : nullptr;
  ex.probe = g->d_tb_probe;
  ex.probe_mid = probe_mid;
  return ex;
}

int ensure_tb_ready(jxf_grid3d* g) {
  if (g->tb < 0) return JXF_OK;
  if (!g->maps_tb_ok || g->maps_tb_cfg != g->tb) TRY(encode_maps_tb(g));
  if (g->tb_built_cfg != g->tb || g->tb_built_chunk != g->tb_chunk) TRY(build_tb_lists(g));
  return JXF_OK;
}

int heuristic_tune(jxf_grid3d* g) {
  // Small grids: smaller tiles and chunks keep >= 2 waves of blocks.
  const long long cells = g->n;
  g->cfg = 0;
  g->x_chunk = cells >= (1LL << 24) ? 64 : (cells >= (1LL << 21) ? 16 : 8);
  g->axis_split = cells >= (1LL << 25) ? 1 : 0;
  return JXF_OK;
}

// JXF_AXIS_SPLIT=0/1 forces the single-axis shell split off / on.
int axis_split_override() {
  const char* e = std::getenv("JXF_AXIS_SPLIT");
  return e ? (std::atoi(e) != 0 ? 1 : 0) : -1;
}

// Time every (config, chunk, axis split) on A -> B launches (the state in A
// and the step counter are untouched, probes off) and keep the fastest.
int autotune(jxf_grid3d* g, cudaStream_t st) {
  // (x-slabs tune apart from whole grids: they take no blocked passes)
  const auto key = std::make_tuple(g->d.nx, g->d.ny, g->d.nz,
                                   g->mode * 4 + (g->kappa ? 1 : 0) + (g->slab ? 2 : 0),
                                   g->cb ? 1 : 0);
  const int split_env = axis_split_override();
  {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      g->cfg = std::get<0>(it->second);
      g->x_chunk = std::get<1>(it->second);
      g->axis_split = std::get<2>(it->second);
      g->tb = std::get<3>(it->second);
      g->tb_chunk = std::get<4>(it->second);
      return JXF_OK;
    }
  }
  // JXF_TB: "off" keeps one step per launch; "cfg,chunk[,split]" pins the
  // two-level blocked launch shape
  const char* tb_env = std::getenv("JXF_TB");
  // (x-slabs take one step per pass: ghost planes are exchanged between steps)
  const bool tb_off = (tb_env && std::strcmp(tb_env, "off") == 0) || g->slab;
  int tfc = -1, tfk = -1, tfs = -1;
  const bool tb_forced = tb_env && !tb_off && !g->slab &&
                         std::sscanf(tb_env, "%d,%d,%d", &tfc, &tfk, &tfs) >= 2 && tfc >= 0 &&
                         tfc < (int)tb_configs().size() && tfk >= 1;
  const char* env = std::getenv("JXF_AUTOTUNE");
  const bool enabled = !(env && env[0] == '0');
  // "cfg,chunk[,split]": pin the launch shape (split defaults to off)
  const char* forced = std::getenv("JXF_LAUNCH");
  int fc = -1, fk = -1, fs = 0;
  if (forced && std::sscanf(forced, "%d,%d,%d", &fc, &fk, &fs) >= 2 && fc >= 0 &&
      fc < (int)tma_configs().size() && fk >= 1) {
    g->cfg = fc;
    g->x_chunk = fk;
    g->axis_split = split_env >= 0 ? split_env : (fs != 0 ? 1 : 0);
    g->tb = tb_forced ? tfc : -1;
    g->tb_chunk = tb_forced ? tfk : 0;
    if (tb_forced && tfs >= 0) g->axis_split = tfs != 0 ? 1 : 0;
    return JXF_OK;
  }
  if (tb_forced) {
    TRY(heuristic_tune(g));
    g->tb = tfc;
    g->tb_chunk = tfk;
    if (tfs >= 0) g->axis_split = tfs != 0 ? 1 : 0;
    if (split_env >= 0) g->axis_split = split_env;
  } else if (!enabled || g->n < (1LL << 18)) {
    TRY(heuristic_tune(g));
    g->tb = -1;
    if (split_env >= 0) g->axis_split = split_env;
  } else {
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    float best = 1e30f;
    int bc = 0, bk = 8, bs = 0;
    // short chunks give small grids more blocks (64^3: 2 planes per block is
    // fastest), long ones cut the warm-up plane share on large grids
    const int chunks[] = {2, 4, 8, 16, 32, 64};
    const bool can_split = g->mode == MODE_CPML && !g->kappa;
    for (int sp = 0; sp < 2; ++sp) {
      if (sp == 1 && !can_split) continue;
      if (split_env >= 0 && sp != split_env) continue;
      for (int ci = 0; ci < (int)tma_configs().size(); ++ci) {
        for (int ch : chunks) {
          if (ch > g->d.nx && ch != 8) continue;
          g->cfg = ci;
          g->x_chunk = ch;
          g->axis_split = sp;
          TRY(encode_maps(g));
          Step3D p = base_params(g);
          set_io(g, p, g->cur, 1 - g->cur);
          p.blk_src_ptr = nullptr;
          p.probe_out = nullptr;
          p.step = 0;
          p.err = g->d_err;
          TRY(launch_step(g, ci, ch, p, g->cur, st));
          // trials of about 2 ms or more (small grids run many steps), best of two
          const int reps = g->n >= (1LL << 25) ? 3 : (g->n >= (1LL << 21) ? 40 : 100);
          float ms = 1e30f;
          for (int trial = 0; trial < 2; ++trial) {
            CUDA_TRY(cudaEventRecord(e0, st));
            for (int r = 0; r < reps; ++r) TRY(launch_step(g, ci, ch, p, g->cur, st));
            CUDA_TRY(cudaEventRecord(e1, st));
            CUDA_TRY(cudaEventSynchronize(e1));
            float t = 0;
            CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
            ms = std::min(ms, t / (float)reps);  // per leapfrog step
          }
          if (ms < best) {
            best = ms;
            bc = ci;
            bk = ch;
            bs = sp;
          }
        }
      }
    }
    // two-level blocked launches: time per leapfrog step = launch time / 2
    int btb = -1, btk = 0, bts = bs;
    if (!tb_off) {
      const int tchunks[] = {8, 16, 32, 64};
      for (int sp = 0; sp < 2; ++sp) {
        if (sp == 1 && !can_split) continue;
        if (split_env >= 0 && sp != split_env) continue;
        for (int ti = 0; ti < (int)tb_configs().size(); ++ti) {
          for (int ch : tchunks) {
            if (ch > g->d.nx && ch != 8) continue;
            g->tb = ti;
            g->tb_chunk = ch;
            g->axis_split = sp;
            TRY(encode_maps_tb(g));
            Step3D p = base_params(g);
            set_io(g, p, g->cur, 1 - g->cur);
            p.blk_src_ptr = nullptr;
            p.probe_out = nullptr;
            p.step = 0;
            p.err = g->d_err;
            TbExtra ex{};
            TRY(launch_tb_step(g, ti, ch, p, ex, g->cur, st));
            const int reps = g->n >= (1LL << 25) ? 2 : (g->n >= (1LL << 21) ? 20 : 50);
            float ms = 1e30f;
            for (int trial = 0; trial < 2; ++trial) {
              CUDA_TRY(cudaEventRecord(e0, st));
              for (int r = 0; r < reps; ++r) TRY(launch_tb_step(g, ti, ch, p, ex, g->cur, st));
              CUDA_TRY(cudaEventRecord(e1, st));
              CUDA_TRY(cudaEventSynchronize(e1));
              float t = 0;
              CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
              ms = std::min(ms, t / (2.0f * (float)reps));  // two leapfrog steps per launch
            }
            if (ms < best) {
              best = ms;
              btb = ti;
              btk = ch;
              bts = sp;
            }
          }
        }
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    g->cfg = bc;
    g->x_chunk = bk;
    g->axis_split = btb >= 0 ? bts : bs;
    g->tb = btb;
    g->tb_chunk = btk;
    g->maps_ok = false;  // maps hold the boxes of the last trial, not of the winner
    g->maps_tb_ok = false;
    g->built_cfg = -1;
    g->tb_built_cfg = -1;
    // The trials wrote only the idle buffer set, which the next real step
    // overwrites before anything reads it.
  }
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune_cache[key] = std::make_tuple(g->cfg, g->x_chunk, g->axis_split, g->tb, g->tb_chunk);
  return JXF_OK;
}

int ensure_tma_ready(jxf_grid3d* g, cudaStream_t st) {
  if (g->cfg < 0) TRY(autotune(g, st));
  if (!g->maps_ok) TRY(encode_maps(g));
  if (!g->src_cell.empty() && (g->built_cfg != g->cfg || g->built_chunk != g->x_chunk))
    TRY(build_tma_sources(g));
  TRY(ensure_tb_ready(g));
  return JXF_OK;
}

}  // namespace

extern "C" {

const char* jxf_last_error(void) { return g_last_error.c_str(); }

int jxf_version(void) { return 100; }

// ---- field viewers (viz_kernels.cuh)
static int slice_args(const float* src, int64_t nu, int64_t nv, int32_t n_frames) {
  if (!src) return fail(JXF_ERR_INVALID, "null slice pointer");
  if (nu <= 0 || nv <= 0 || n_frames <= 0)
    return fail(JXF_ERR_INVALID, "empty slice (%lld x %lld, %d frames)", (long long)nu,
                (long long)nv, n_frames);
  return JXF_OK;
}

int jxf_slice_absmax(const float* src, int64_t nu, int64_t nv, int64_t su, int64_t sv,
                     int32_t n_frames, int64_t sf, float* out, void* stream) {
  TRY(slice_args(src, nu, nv, n_frames));
  if (!out) return fail(JXF_ERR_INVALID, "null output");
  cudaStream_t st = (cudaStream_t)stream;
  const long long total = (long long)n_frames * nu * nv;
  CUDA_TRY(cudaMemsetAsync(out, 0, sizeof(float), st));
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 8);
  jxf::k_slice_absmax<<<blocks, 256, 0, st>>>(src, nu, nv, su, sv, sf, total, out);
  CUDA_TRY(cudaGetLastError());
  return JXF_OK;
}

int jxf_slice_rgb(const float* src, int64_t nu, int64_t nv, int64_t su, int64_t sv,
                  int32_t n_frames, int64_t sf, const float* vmax_dev, float vmax,
                  const uint8_t* lut, uint8_t* out, void* stream) {
  TRY(slice_args(src, nu, nv, n_frames));
  if (!lut || !out) return fail(JXF_ERR_INVALID, "null colour table or output");
  cudaStream_t st = (cudaStream_t)stream;
  const long long total = (long long)n_frames * nu * nv;
  const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 16);
  jxf::k_slice_rgb<<<blocks, 256, 0, st>>>(src, nu, nv, su, sv, sf, total, vmax_dev, vmax, lut,
                                           out);
  CUDA_TRY(cudaGetLastError());
  return JXF_OK;
}

static int create3d(const jxf_grid3d_desc& d, int gnx, int gx0, int x_lo, int x_hi, bool slab,
                    jxf_grid3d** out);

int jxf_grid3d_create(const jxf_grid3d_desc* desc, jxf_grid3d** out) {
  if (!desc || !out) return fail(JXF_ERR_INVALID, "null argument");
  *out = nullptr;
  return create3d(*desc, desc->nx, 0, 0, desc->nx, false, out);
}

int jxf_grid3d_create_slab(const jxf_grid3d_desc* desc, int32_t x0, int32_t x1,
                           jxf_grid3d** out) {
  if (!desc || !out) return fail(JXF_ERR_INVALID, "null argument");
  *out = nullptr;
  if (x0 < 0 || x1 > desc->nx || x1 - x0 < 1)
    return fail(JXF_ERR_INVALID, "slab [%d, %d) outside the grid's %d planes", x0, x1, desc->nx);
  if (desc->boundary == JXF_BND_PERIODIC)
    return fail(JXF_ERR_INVALID, "x-slab decomposition does not support PERIODIC boundaries");
  jxf_grid3d_desc d = *desc;
  d.nx = x1 - x0 + 2;  // owned planes plus one ghost plane on each side
  return create3d(d, desc->nx, x0 - 1, 1, x1 - x0 + 1, true, out);
}

static int create3d_impl(const jxf_grid3d_desc& d, int gnx, int gx0, int x_lo, int x_hi,
                         bool slab, jxf_grid3d** out);

static int create3d(const jxf_grid3d_desc& d, int gnx, int gx0, int x_lo, int x_hi, bool slab,
                    jxf_grid3d** out) {
  const char* e = std::getenv("JXF_FAULT_ALLOC_AFTER");
  g_alloc_budget = (e && *e) ? std::max(0LL, std::atoll(e)) : -1;
  const int rc = create3d_impl(d, gnx, gx0, x_lo, x_hi, slab, out);
  g_alloc_budget = -1;
  return rc;
}

static int create3d_impl(const jxf_grid3d_desc& d, int gnx, int gx0, int x_lo, int x_hi,
                         bool slab, jxf_grid3d** out) {
  if (d.nx < 2 || d.ny < 2 || d.nz < 2)
    return fail(JXF_ERR_INVALID, "grid must be at least 2 cells per axis, got %dx%dx%d", d.nx, d.ny,
                d.nz);
  if ((long long)d.nx * d.ny * d.nz > (1LL << 36))
    return fail(JXF_ERR_INVALID, "grid too large");
  if (!(d.dx > 0)) return fail(JXF_ERR_INVALID, "dx must be positive");
  if (d.pml_layers < 0) return fail(JXF_ERR_INVALID, "pml_layers must be >= 0");
  if (d.boundary != JXF_BND_ABSORBING && d.boundary != JXF_BND_PERIODIC &&
      d.boundary != JXF_BND_PEC && d.boundary != JXF_BND_CPML)
    return fail(JXF_ERR_INVALID, "unsupported 3D boundary %d", d.boundary);
  if (d.boundary == JXF_BND_CPML && !(d.cpml_r0 > 0 && d.cpml_r0 < 1))
    return fail(JXF_ERR_INVALID, "cpml_r0 must be in (0, 1)");
  DeviceGuard dg(d.device);
  if (!dg.ok) return fail(JXF_ERR_CUDA, "cannot select device %d", d.device);

  jxf_grid3d* g = new jxf_grid3d();
  g->d = d;
  g->n = (long long)d.nx * d.ny * d.nz;
  g->gnx = gnx;
  g->gx0 = gx0;
  g->x_lo = x_lo;
  g->x_hi = x_hi;
  g->slab = slab;
  g->dt = d.dt > 0 ? d.dt : 0.99 * d.dx / (kC0 * std::sqrt(3.0));  // fdtd3d.py:190-192
  g->coef_h = g->dt / (kMu0 * d.dx);                                 // fdtd3d.py:223
  g->coef_e = g->dt / (kEps0 * d.dx);                                // fdtd3d.py:224
  g->mode = d.boundary == JXF_BND_PERIODIC ? MODE_PERIODIC
            : d.boundary == JXF_BND_CPML   ? MODE_CPML
                                           : MODE_ABSORB;
  const bool tma_ok = (d.nz % 4 == 0) && g->mode != MODE_PERIODIC;
  if (d.path == JXF_PATH_TMA && !tma_ok) {
    delete g;
    return fail(JXF_ERR_INVALID, "TMA path needs nz %% 4 == 0 and a non-periodic boundary");
  }
  g->path = (d.path == JXF_PATH_GENERIC || !tma_ok) ? JXF_PATH_GENERIC : JXF_PATH_TMA;
  {
    const char* e = std::getenv("JXF_PDL");
    g->use_pdl = !(e && e[0] == '0');
  }
  if (g->mode == MODE_CPML && g->path == JXF_PATH_TMA) {
    // the TMA kernel addresses psi slabs with 32-bit offsets
    const long long P2 = 2LL * (d.pml_layers + 1);
    const long long big = (long long)std::max(d.nx, std::max(d.ny, d.nz));
    const long long mid = (long long)d.nx * d.ny * d.nz / big;
    if (std::min(P2, big) * mid >= (1LL << 31) || (long long)d.ny * d.nz >= (1LL << 31)) {
      if (d.path == JXF_PATH_TMA) {
        delete g;
        return fail(JXF_ERR_INVALID, "grid too large for 32-bit CPML slab offsets on the TMA path");
      }
      g->path = JXF_PATH_GENERIC;
    }
  }

  auto cleanup_fail = [&](int rc) {
    jxf_grid3d_destroy(g);
    return rc;
  };
  int rc;
  for (int s = 0; s < 2; ++s)
    for (int k = 0; k < 6; ++k) {
      if (s == 1 && g->path == JXF_PATH_GENERIC) break;
      if ((rc = dmalloc(&g->f[s][k], (size_t)g->n, &g->bytes)) != JXF_OK) return cleanup_fail(rc);
      cudaMemset(g->f[s][k], 0, (size_t)g->n * 4);
    }
  if (g->path == JXF_PATH_GENERIC)
    for (int k = 0; k < 6; ++k) g->f[1][k] = g->f[0][k];

  // coefficient tables along x cover the whole (global) axis
  const int dims[3] = {gnx, d.ny, d.nz};
  // damping tables (ones for PEC / CPML / PERIODIC)
  for (int ax = 0; ax < 3; ++ax) {
    std::vector<float> t = (d.boundary == JXF_BND_ABSORBING)
                               ? damping_table(dims[ax], d.pml_layers, d.dx, g->dt, 3)
                               : std::vector<float>(dims[ax], 1.0f);
    if ((rc = upload(&g->damp[ax], t, &g->bytes)) != JXF_OK) return cleanup_fail(rc);
  }
  if (g->mode == MODE_CPML) {
    const double m = d.cpml_order > 0 ? d.cpml_order : 3.0;
    const double kmax = d.cpml_kappa_max >= 1.0 ? d.cpml_kappa_max : 1.0;
    g->kappa = kmax > 1.0;
    for (int ax = 0; ax < 3; ++ax) {
      std::vector<float> t[TAB_COUNT];
      cpml_tables(dims[ax], d.pml_layers, d.dx, g->dt, m, d.cpml_r0, kmax, d.cpml_alpha_max, t);
      for (int k = 0; k < TAB_COUNT; ++k)
        if ((rc = upload(&g->tab[ax][k], t[k], &g->bytes)) != JXF_OK) return cleanup_fail(rc);
      const int P = d.pml_layers + 1;
      if (2 * P >= dims[ax]) {
        g->P[ax] = -1;
        g->L[ax] = dims[ax];
      } else {
        g->P[ax] = P;
        g->L[ax] = 2 * P;
      }
    }
    const size_t sz_x = (size_t)g->L[0] * d.ny * d.nz;
    const size_t sz_y = (size_t)d.nx * g->L[1] * d.nz;
    const size_t sz_z = (size_t)d.nx * d.ny * g->L[2];
    const int axis_of[PSI_COUNT] = {1, 2, 2, 0, 0, 1, 1, 2, 2, 0, 0, 1};
    for (int s = 0; s < 2; ++s)
      for (int k = 0; k < PSI_COUNT; ++k) {
        if (s == 1 && g->path == JXF_PATH_GENERIC) {
          g->psi[1][k] = g->psi[0][k];
          continue;
        }
        const size_t sz = axis_of[k] == 0 ? sz_x : (axis_of[k] == 1 ? sz_y : sz_z);
        if ((rc = dmalloc(&g->psi[s][k], sz, &g->bytes)) != JXF_OK) return cleanup_fail(rc);
        cudaMemset(g->psi[s][k], 0, sz * 4);
      }
  } else {
    // tables are dereferenced only in CPML mode; keep valid pointers anyway
    for (int ax = 0; ax < 3; ++ax)
      for (int k = 0; k < TAB_COUNT; ++k) g->tab[ax][k] = g->damp[ax];
  }
  if ((rc = dmalloc(&g->d_err, 4, &g->bytes)) != JXF_OK) return cleanup_fail(rc);
  if ((rc = dmalloc(&g->d_count, 1, &g->bytes)) != JXF_OK) return cleanup_fail(rc);
  cudaMemset(g->d_err, 0, 16);
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess)
    return cleanup_fail(fail(JXF_ERR_CUDA, "initialisation failed: %s", cudaGetErrorString(e)));
  *out = g;
  return JXF_OK;
}

int jxf_grid3d_destroy(jxf_grid3d* g) {
  if (!g) return JXF_OK;
  DeviceGuard dg(g->d.device);
  const bool shared_f = g->path == JXF_PATH_GENERIC;
  for (int s = 0; s < 2; ++s)
    for (int k = 0; k < 6; ++k) {
      if (s == 1 && shared_f) break;
      dfree(g->f[s][k]);
    }
  const bool cpml = g->mode == MODE_CPML;
  for (int s = 0; s < 2; ++s)
    for (int k = 0; k < PSI_COUNT; ++k) {
      if (s == 1 && shared_f) break;
      dfree(g->psi[s][k]);
    }
  if (cpml)
    for (int ax = 0; ax < 3; ++ax)
      for (int k = 0; k < TAB_COUNT; ++k) dfree(g->tab[ax][k]);
  for (int ax = 0; ax < 3; ++ax) dfree(g->damp[ax]);
  dfree(g->cb);
  band_release(g->band);
  dfree(g->d_cells);
  dfree(g->d_terms);
  dfree(g->d_entries);
  dfree(g->d_blk_ptr);
  dfree(g->d_shell);
  for (int a = 0; a < 3; ++a) dfree(g->d_shell_ax[a]);
  dfree(g->d_inner);
  dfree(g->d_tb_src);
  dfree(g->d_tb_src_ptr);
  dfree(g->d_tb_probe);
  dfree(g->d_tb_probe_ptr);
  dfree(g->d_tb_shell);
  for (int a = 0; a < 6; ++a) dfree(g->d_tb_shell_ax[a]);
  dfree(g->d_tb_inner);
  dfree(g->adj_ck);
  dfree(g->adj_sg);
  dfree(g->adj_l);
  dfree(g->adj_g);
  dfree(g->d_wave);
  dfree(g->d_probe_cell);
  dfree(g->d_probe_comp);
  dfree(g->d_err);
  dfree(g->d_count);
  delete g;
  return JXF_OK;
}

int jxf_grid3d_get_info(const jxf_grid3d* g, jxf_grid3d_info* out) {
  if (!g || !out) return fail(JXF_ERR_INVALID, "null argument");
  out->dt = g->dt;
  out->coef_h = g->coef_h;
  out->coef_e = g->coef_e;
  out->step = g->step;
  out->path = g->path;
  if (g->path == JXF_PATH_TMA && g->cfg >= 0) {
    const TmaConfig& c = tma_configs()[g->cfg];
    out->tile_z = c.tz;
    out->tile_y = c.ty;
    out->rows_per_thread = c.ry;
    out->stages = c.stages;
    out->x_chunk = g->x_chunk;
  } else {
    out->tile_z = out->tile_y = out->rows_per_thread = out->stages = out->x_chunk = 0;
  }
  out->device_bytes = g->bytes;
  out->shell_blocks = g->n_shell + g->n_shell_ax[0] + g->n_shell_ax[1] + g->n_shell_ax[2];
  out->interior_blocks = g->n_inner;
  out->tma_config = g->path == JXF_PATH_TMA ? g->cfg : -1;
  out->axis_split = g->axis_split;
  out->blocked_config = g->path == JXF_PATH_TMA ? g->tb : -1;
  out->blocked_x_chunk = g->path == JXF_PATH_TMA && g->tb >= 0 ? g->tb_chunk : 0;
  if (g->path == JXF_PATH_TMA && g->tb >= 0)
    out->blocked_kernels_per_pass =
        g->mode != MODE_CPML || g->tb_split_cfg < 0
            ? 1
            : (g->n_tb_shell > 0 ? 1 : 0) + (g->n_tb_inner > 0 ? 1 : 0) +
                  (g->n_tb_shell_ax[0] > 0 ? 1 : 0) + (g->n_tb_shell_ax[1] > 0 ? 1 : 0) +
                  (g->n_tb_shell_ax[2] > 0 ? 1 : 0) + (g->n_tb_shell_ax[3] > 0 ? 1 : 0) +
                  (g->n_tb_shell_ax[4] > 0 ? 1 : 0) + (g->n_tb_shell_ax[5] > 0 ? 1 : 0);
  else
    out->blocked_kernels_per_pass = 0;
  if (g->path == JXF_PATH_GENERIC)
    out->kernels_per_step = 2 + (g->n_cells > 0 ? 1 : 0);
  else if (g->mode == MODE_CPML && g->split_cfg >= 0)
    out->kernels_per_step = (g->n_shell > 0 ? 1 : 0) + (g->n_inner > 0 ? 1 : 0) +
                            (g->n_shell_ax[0] > 0 ? 1 : 0) + (g->n_shell_ax[1] > 0 ? 1 : 0) +
                            (g->n_shell_ax[2] > 0 ? 1 : 0);
  else
    out->kernels_per_step = 1;
  return JXF_OK;
}

// Fix the TMA launch shape (cfg index into the registry, planes per block);
// cfg < 0 re-enables autotuning.
int jxf_grid3d_set_launch(jxf_grid3d* g, int32_t cfg, int32_t x_chunk) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  if (g->path != JXF_PATH_TMA) return fail(JXF_ERR_INVALID, "grid does not use the TMA path");
  if (cfg >= (int)tma_configs().size()) return fail(JXF_ERR_INVALID, "cfg out of range");
  if (cfg >= 0 && x_chunk < 1) return fail(JXF_ERR_INVALID, "x_chunk must be >= 1");
  g->cfg = cfg;
  g->x_chunk = x_chunk;
  g->maps_ok = false;
  g->built_cfg = -1;
  return JXF_OK;
}

int jxf_num_blocked_configs(void) { return (int)tb_configs().size(); }

int jxf_grid3d_set_blocked(jxf_grid3d* g, int32_t cfg, int32_t x_chunk) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  if (g->path != JXF_PATH_TMA) return fail(JXF_ERR_INVALID, "grid does not use the TMA path");
  if (cfg >= (int)tb_configs().size()) return fail(JXF_ERR_INVALID, "blocked cfg out of range");
  if (cfg >= 0 && g->slab)
    return fail(JXF_ERR_INVALID, "x-slab grids take one step per pass (no blocked passes)");
  if (cfg >= 0 && x_chunk < 1) return fail(JXF_ERR_INVALID, "x_chunk must be >= 1");
  if (g->cfg < 0) TRY(heuristic_tune(g));  // one-step shape for odd remainders
  g->tb = cfg < 0 ? -1 : cfg;
  g->tb_chunk = cfg < 0 ? 0 : x_chunk;
  g->maps_tb_ok = false;
  g->tb_built_cfg = -1;
  g->tb_split_cfg = -1;
  return JXF_OK;
}

int jxf_grid3d_set_axis_split(jxf_grid3d* g, int32_t on) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  g->axis_split = on ? 1 : 0;
  return JXF_OK;
}

int jxf_num_tma_configs(void) { return (int)tma_configs().size(); }

static __global__ void k_cb_from_eps(const float* eps, float* cb, float coef, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    cb[i] = __fdiv_rn(coef, eps[i]);
}

int jxf_grid3d_set_eps_host(jxf_grid3d* g, const double* eps_r) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  DeviceGuard dg(g->d.device);
  if (!eps_r) {
    dfree(g->cb);
    g->maps_ok = false;
    g->maps_tb_ok = false;
    return JXF_OK;
  }
  std::vector<float> cb((size_t)g->n);
  for (long long i = 0; i < g->n; ++i) {
    // +inf marks a perfect electric conductor cell: Cb = 0 keeps its E at zero
    if (!(eps_r[i] > 0) || std::isnan(eps_r[i]))
      return fail(JXF_ERR_INVALID, "eps_r must be positive (or +inf) (cell %lld)", i);
    cb[i] = (float)(g->coef_e / eps_r[i]);  // fdtd3d.py:299 (dt_eps_dx / eps_r), FP64 then round
  }
  TRY(upload(&g->cb, cb, &g->bytes));
  g->maps_ok = false;
  g->maps_tb_ok = false;
  return JXF_OK;
}

int jxf_grid3d_set_eps_device(jxf_grid3d* g, const float* eps_r, void* stream) {
  if (!g || !eps_r) return fail(JXF_ERR_INVALID, "null argument");
  DeviceGuard dg(g->d.device);
  if (!g->cb) {
    TRY(dmalloc(&g->cb, (size_t)g->n, &g->bytes));
  }
  k_cb_from_eps<<<592, 256, 0, (cudaStream_t)stream>>>(eps_r, g->cb, (float)g->coef_e, g->n);
  CUDA_TRY(cudaGetLastError());
  g->maps_ok = false;
  g->maps_tb_ok = false;
  return JXF_OK;
}

int jxf_grid3d_set_sources(jxf_grid3d* g, int32_t n, const int64_t* cell, const int32_t* comp,
                           const float* amplitude, const int32_t* wave_id) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  if (n < 0 || (n > 0 && (!cell || !comp || !amplitude || !wave_id)))
    return fail(JXF_ERR_INVALID, "bad source arrays");
  DeviceGuard dg(g->d.device);
  for (int i = 0; i < n; ++i) {
    if (!cells_ok(g, cell[i])) return fail(JXF_ERR_INVALID, "source %d: cell out of grid", i);
    if (comp[i] < 0 || comp[i] > 2) return fail(JXF_ERR_INVALID, "source %d: comp must be 0..2", i);
    if (wave_id[i] < 0) return fail(JXF_ERR_INVALID, "source %d: negative wave id", i);
  }
  g->src_cell.assign(cell, cell + n);
  g->src_comp.assign(comp, comp + n);
  g->src_amp.assign(amplitude, amplitude + n);
  g->src_wave.assign(wave_id, wave_id + n);
  TRY(build_generic_sources(g));
  g->built_cfg = -1;
  g->tb_built_cfg = -1;
  return JXF_OK;
}

int jxf_grid3d_set_waveforms(jxf_grid3d* g, int32_t n_waves, int64_t n_samples,
                             const float* samples) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  if (n_waves < 0 || n_samples < 0 || (n_waves * n_samples > 0 && !samples))
    return fail(JXF_ERR_INVALID, "bad waveform table");
  DeviceGuard dg(g->d.device);
  std::vector<float> v(samples, samples + (size_t)n_waves * n_samples);
  TRY(upload(&g->d_wave, v, &g->bytes));
  g->n_waves = n_waves;
  g->wave_len = n_samples;
  return JXF_OK;
}

int jxf_grid3d_set_probes(jxf_grid3d* g, int32_t n, const int64_t* cell, const int32_t* comp) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  if (n < 0 || (n > 0 && (!cell || !comp))) return fail(JXF_ERR_INVALID, "bad probe arrays");
  DeviceGuard dg(g->d.device);
  for (int i = 0; i < n; ++i) {
    if (!cells_ok(g, cell[i])) return fail(JXF_ERR_INVALID, "probe %d: cell out of grid", i);
    if (comp[i] < 0 || comp[i] > 5) return fail(JXF_ERR_INVALID, "probe %d: comp must be 0..5", i);
  }
  std::vector<long long> c(cell, cell + n);
  std::vector<int> k(comp, comp + n);
  TRY(upload(&g->d_probe_cell, c, &g->bytes));
  TRY(upload(&g->d_probe_comp, k, &g->bytes));
  g->n_probes = n;
  g->probe_cell_h = c;
  g->probe_comp_h = k;
  g->tb_built_cfg = -1;
  return JXF_OK;
}

static int gather_probes(jxf_grid3d* g, int set, float* out, cudaStream_t st) {
  if (g->n_probes == 0 || !out) return JXF_OK;
  FieldPtrs6 fp;
  for (int k = 0; k < 6; ++k) fp.f[k] = g->f[set][k];
  k_probe_gather<<<(g->n_probes + 127) / 128, 128, 0, st>>>(fp, g->d_probe_cell, g->d_probe_comp,
                                                           g->n_probes, out);
  CUDA_TRY(cudaGetLastError());
  return JXF_OK;
}

int jxf_grid3d_step(jxf_grid3d* g, int32_t n_steps, float* probe_out, void* stream) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  if (g->slab && g->path != JXF_PATH_TMA)
    return fail(JXF_ERR_INVALID, "x-slab grids on the generic path advance with "
                "jxf_grid3d_half_step (ghost exchange)");
  if (g->slab && n_steps > 1)
    return fail(JXF_ERR_INVALID, "an x-slab grid takes one step per call (its ghost planes are "
                "exchanged between steps)");
  if (n_steps < 0) return fail(JXF_ERR_INVALID, "n_steps must be >= 0");
  if (n_steps == 0) return JXF_OK;
  if (!g->src_cell.empty()) {
    int max_w = 0;
    for (int w : g->src_wave) max_w = std::max(max_w, w);
    if (max_w >= g->n_waves)
      return fail(JXF_ERR_INVALID, "source wave id %d has no waveform row", max_w);
    if (g->step + n_steps > g->wave_len)
      return fail(JXF_ERR_INVALID, "waveform table covers %lld steps, need %lld", g->wave_len,
                  g->step + n_steps);
  }
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  Step3D p = base_params(g);
  const int np = g->n_probes;
  if (g->path == JXF_PATH_TMA) {
    TRY(ensure_tma_ready(g, st));
    p.blk_src_ptr = g->src_cell.empty() ? nullptr : g->d_blk_ptr;
    p.src = g->d_entries;
    for (int k = 0; k < n_steps;) {
      set_io(g, p, g->cur, 1 - g->cur);
      p.step = g->step;
      p.probe_out = (probe_out && np > 0 && k >= 1) ? probe_out + (size_t)(k - 1) * np : nullptr;
      // (a learned band corrects the state between every two steps, so its
      // grids take one step per pass)
      if (g->tb >= 0 && !g->band.band && n_steps - k >= 2) {
        // two steps in one pass; the state after the first is recorded by
        // the probe cells' owner blocks
        const TbExtra ex = tb_extra(g, (probe_out && np > 0) ? probe_out + (size_t)k * np : nullptr);
        TRY(launch_tb_step(g, g->tb, g->tb_chunk, p, ex, g->cur, st));
        g->cur ^= 1;
        g->step += 2;
        k += 2;
        continue;
      }
      TRY(launch_step(g, g->cfg, g->x_chunk, p, g->cur, st));
      g->cur ^= 1;
      g->step++;
      ++k;
      if (g->band.band) TRY(band_launch(g->band, st, g->cur));
    }
    if (probe_out && np > 0) TRY(gather_probes(g, g->cur, probe_out + (size_t)(n_steps - 1) * np, st));
  } else {
    const int threads = 256;
    const long long blocks_needed = (g->n + threads - 1) / threads;
    const int blocks = (int)std::min<long long>(blocks_needed, 148LL * 16);
    for (int k = 0; k < n_steps; ++k) {
      set_io(g, p, 0, 0);
      p.step = g->step;
      switch (g->mode) {
        case MODE_PERIODIC:
          jxf::k3d_generic_h<MODE_PERIODIC><<<blocks, threads, 0, st>>>(p);
          jxf::k3d_generic_e<MODE_PERIODIC><<<blocks, threads, 0, st>>>(p);
          break;
        case MODE_CPML:
          jxf::k3d_generic_h<MODE_CPML><<<blocks, threads, 0, st>>>(p);
          jxf::k3d_generic_e<MODE_CPML><<<blocks, threads, 0, st>>>(p);
          break;
        default:
          jxf::k3d_generic_h<MODE_ABSORB><<<blocks, threads, 0, st>>>(p);
          jxf::k3d_generic_e<MODE_ABSORB><<<blocks, threads, 0, st>>>(p);
          break;
      }
      CUDA_TRY(cudaGetLastError());
      if (g->n_cells > 0) {
        k3d_sources<<<(g->n_cells + 127) / 128, 128, 0, st>>>(
            g->f[0][0], g->f[0][1], g->f[0][2], g->d_cells, g->n_cells, g->d_terms, g->d_wave,
            g->wave_len, g->step);
        CUDA_TRY(cudaGetLastError());
      }
      if (g->band.band) TRY(band_launch(g->band, st));
      if (probe_out && np > 0) TRY(gather_probes(g, 0, probe_out + (size_t)k * np, st));
      g->step++;
    }
  }
  return JXF_OK;
}

}  // extern "C"

namespace {
// Soft sources of the cells whose plane lies in [plo, phi) (slab half-steps
// split into a boundary plane and the rest).
__global__ void k3d_sources_planes(float* ex, float* ey, float* ez, const SrcCell* cells,
                                   int n_cells, const SrcTerm* terms, const float* wave,
                                   long long wave_len, long long step, long long plane, int plo,
                                   int phi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_cells) return;
  const SrcCell c = cells[i];
  const long long x = c.cell / plane;
  if (x < plo || x >= phi) return;
  float* f = c.comp == 0 ? ex : (c.comp == 1 ? ey : ez);
  float v = f[c.cell];
  for (int k = 0; k < c.count; ++k) {
    const SrcTerm t = terms[c.first + k];
    v = fadd(v, fmul(t.amp, wave[(long long)t.wave * wave_len + step]));
  }
  f[c.cell] = v;
}
}  // namespace

extern "C" {

int jxf_grid3d_half_step_part(jxf_grid3d* g, int32_t half, int32_t part, float* probe_row,
                              void* stream) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  if (!g->slab) return fail(JXF_ERR_INVALID, "half steps are for x-slab grids");
  if (g->path != JXF_PATH_GENERIC)
    return fail(JXF_ERR_INVALID, "half steps run on generic-path x-slabs (a TMA x-slab takes "
                "whole steps: jxf_grid3d_step)");
  if (half != 0 && half != 1) return fail(JXF_ERR_INVALID, "half must be 0 (H) or 1 (E)");
  if (part < 0 || part > 2) return fail(JXF_ERR_INVALID, "part must be 0, 1 or 2");
  if (part == 0) return jxf_grid3d_half_step(g, half, probe_row, stream);
  if (g->x_hi - g->x_lo < 2)
    return fail(JXF_ERR_INVALID, "a split half-step needs at least two owned planes");
  if (half == 1 && !g->src_cell.empty()) {
    int max_w = 0;
    for (int w : g->src_wave) max_w = std::max(max_w, w);
    if (max_w >= g->n_waves || g->step + 1 > g->wave_len)
      return fail(JXF_ERR_INVALID, "waveform table does not cover step %lld", g->step);
  }
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  Step3D p = base_params(g);
  set_io(g, p, 0, 0);
  p.step = g->step;
  // the plane this half-step hands to a neighbour: H of the last owned plane
  // (the next rank's E needs it), E of the first owned plane (the previous
  // rank's H needs it); part 2 is the rest of the owned planes
  const int bplane = half == 0 ? g->x_hi - 1 : g->x_lo;
  if (part == 1) {
    p.x_lo = bplane;
    p.x_hi = bplane + 1;
  } else if (half == 0) {
    p.x_hi = g->x_hi - 1;
  } else {
    p.x_lo = g->x_lo + 1;
  }
  const int threads = 256;
  const long long owned = (long long)(p.x_hi - p.x_lo) * g->d.ny * g->d.nz;
  const int blocks = (int)std::min<long long>((owned + threads - 1) / threads, 148LL * 16);
  if (half == 0) {
    if (g->mode == MODE_CPML)
      jxf::k3d_generic_h<MODE_CPML><<<blocks, threads, 0, st>>>(p);
    else
      jxf::k3d_generic_h<MODE_ABSORB><<<blocks, threads, 0, st>>>(p);
    CUDA_TRY(cudaGetLastError());
    return JXF_OK;
  }
  if (g->mode == MODE_CPML)
    jxf::k3d_generic_e<MODE_CPML><<<blocks, threads, 0, st>>>(p);
  else
    jxf::k3d_generic_e<MODE_ABSORB><<<blocks, threads, 0, st>>>(p);
  CUDA_TRY(cudaGetLastError());
  if (g->n_cells > 0) {
    k3d_sources_planes<<<(g->n_cells + 127) / 128, 128, 0, st>>>(
        g->f[0][0], g->f[0][1], g->f[0][2], g->d_cells, g->n_cells, g->d_terms, g->d_wave,
        g->wave_len, g->step, (long long)g->d.ny * g->d.nz, p.x_lo, p.x_hi);
    CUDA_TRY(cudaGetLastError());
  }
  if (part == 2) {  // the E half-step ends with its second part
    if (probe_row && g->n_probes > 0) TRY(gather_probes(g, 0, probe_row, st));
    g->step++;
  }
  return JXF_OK;
}

int jxf_grid3d_half_step(jxf_grid3d* g, int32_t half, float* probe_row, void* stream) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  if (!g->slab) return fail(JXF_ERR_INVALID, "half steps are for x-slab grids");
  if (g->path != JXF_PATH_GENERIC)
    return fail(JXF_ERR_INVALID, "half steps run on generic-path x-slabs (a TMA x-slab takes "
                "whole steps: jxf_grid3d_step)");
  if (half != 0 && half != 1) return fail(JXF_ERR_INVALID, "half must be 0 (H) or 1 (E)");
  if (half == 1 && !g->src_cell.empty()) {
    int max_w = 0;
    for (int w : g->src_wave) max_w = std::max(max_w, w);
    if (max_w >= g->n_waves || g->step + 1 > g->wave_len)
      return fail(JXF_ERR_INVALID, "waveform table does not cover step %lld", g->step);
  }
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  Step3D p = base_params(g);
  set_io(g, p, 0, 0);
  p.step = g->step;
  const int threads = 256;
  const long long owned = (long long)(g->x_hi - g->x_lo) * g->d.ny * g->d.nz;
  const int blocks = (int)std::min<long long>((owned + threads - 1) / threads, 148LL * 16);
  if (half == 0) {
    if (g->mode == MODE_CPML)
      jxf::k3d_generic_h<MODE_CPML><<<blocks, threads, 0, st>>>(p);
    else
      jxf::k3d_generic_h<MODE_ABSORB><<<blocks, threads, 0, st>>>(p);
    CUDA_TRY(cudaGetLastError());
    return JXF_OK;
  }
  if (g->mode == MODE_CPML)
    jxf::k3d_generic_e<MODE_CPML><<<blocks, threads, 0, st>>>(p);
  else
    jxf::k3d_generic_e<MODE_ABSORB><<<blocks, threads, 0, st>>>(p);
  CUDA_TRY(cudaGetLastError());
  if (g->n_cells > 0) {
    k3d_sources<<<(g->n_cells + 127) / 128, 128, 0, st>>>(g->f[0][0], g->f[0][1], g->f[0][2],
                                                           g->d_cells, g->n_cells, g->d_terms,
                                                           g->d_wave, g->wave_len, g->step);
    CUDA_TRY(cudaGetLastError());
  }
  if (probe_row && g->n_probes > 0) TRY(gather_probes(g, 0, probe_row, st));
  g->step++;
  return JXF_OK;
}

int jxf_grid3d_plane(jxf_grid3d* g, int32_t comp, int32_t plane, float* buf, int32_t to_buf,
                     void* stream) {
  if (!g || !buf) return fail(JXF_ERR_INVALID, "null argument");
  if (comp < 0 || comp > 5) return fail(JXF_ERR_INVALID, "comp must be 0..5");
  if (plane < 0 || plane >= g->d.nx) return fail(JXF_ERR_INVALID, "plane %d out of range", plane);
  DeviceGuard dg(g->d.device);
  const size_t pl = (size_t)g->d.ny * g->d.nz;
  float* f = g->f[g->cur][comp] + (size_t)plane * pl;
  CUDA_TRY(cudaMemcpyAsync(to_buf ? buf : f, to_buf ? f : buf, pl * 4, cudaMemcpyDeviceToDevice,
                           (cudaStream_t)stream));
  return JXF_OK;
}

int jxf_grid3d_reset(jxf_grid3d* g, void* stream) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  const int sets = g->path == JXF_PATH_GENERIC ? 1 : 2;
  for (int s = 0; s < sets; ++s) {
    for (int k = 0; k < 6; ++k) CUDA_TRY(cudaMemsetAsync(g->f[s][k], 0, (size_t)g->n * 4, st));
    if (g->mode == MODE_CPML) {
      const size_t sz_x = (size_t)g->L[0] * g->d.ny * g->d.nz;
      const size_t sz_y = (size_t)g->d.nx * g->L[1] * g->d.nz;
      const size_t sz_z = (size_t)g->d.nx * g->d.ny * g->L[2];
      const int axis_of[PSI_COUNT] = {1, 2, 2, 0, 0, 1, 1, 2, 2, 0, 0, 1};
      for (int k = 0; k < PSI_COUNT; ++k) {
        const size_t sz = axis_of[k] == 0 ? sz_x : (axis_of[k] == 1 ? sz_y : sz_z);
        CUDA_TRY(cudaMemsetAsync(g->psi[s][k], 0, sz * 4, st));
      }
    }
  }
  g->cur = 0;
  g->step = 0;
  return JXF_OK;
}

int jxf_grid3d_field_ptr(jxf_grid3d* g, int32_t comp, float** out) {
  if (!g || !out) return fail(JXF_ERR_INVALID, "null argument");
  if (comp < 0 || comp > 5) return fail(JXF_ERR_INVALID, "comp must be 0..5");
  *out = g->f[g->cur][comp];
  return JXF_OK;
}

int jxf_grid3d_get_field(jxf_grid3d* g, int32_t comp, float* dst, int32_t dst_is_host,
                         void* stream) {
  if (!g || !dst) return fail(JXF_ERR_INVALID, "null argument");
  if (comp < 0 || comp > 5) return fail(JXF_ERR_INVALID, "comp must be 0..5");
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(cudaMemcpyAsync(dst, g->f[g->cur][comp], (size_t)g->n * 4,
                           dst_is_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, st));
  if (dst_is_host) CUDA_TRY(cudaStreamSynchronize(st));
  return JXF_OK;
}

int jxf_grid3d_set_field(jxf_grid3d* g, int32_t comp, const float* src, int32_t src_is_host,
                         void* stream) {
  if (!g || !src) return fail(JXF_ERR_INVALID, "null argument");
  if (comp < 0 || comp > 5) return fail(JXF_ERR_INVALID, "comp must be 0..5");
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(cudaMemcpyAsync(g->f[g->cur][comp], src, (size_t)g->n * 4,
                           src_is_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st));
  if (src_is_host) CUDA_TRY(cudaStreamSynchronize(st));
  return JXF_OK;
}

int jxf_grid3d_snapshot(jxf_grid3d* g, float* dst, void* stream) {
  if (!g || !dst) return fail(JXF_ERR_INVALID, "null argument");
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  for (int k = 0; k < 6; ++k)
    CUDA_TRY(cudaMemcpyAsync(dst + (size_t)k * g->n, g->f[g->cur][k], (size_t)g->n * 4,
                             cudaMemcpyDeviceToDevice, st));
  return JXF_OK;
}

int jxf_grid3d_check_error(jxf_grid3d* g, void* stream) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  int h[4] = {0, 0, 0, 0};
  CUDA_TRY(cudaMemcpyAsync(h, g->d_err, 16, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  CUDA_TRY(cudaGetLastError());
  if (h[0] != 0) {
    CUDA_TRY(cudaMemsetAsync(g->d_err, 0, 16, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    if (h[0] & ERR_TIMEOUT_BASE)
      return fail(JXF_ERR_TIMEOUT,
                  "a staged copy did not arrive within the wait limit (block %d, plane index %d, "
                  "copies issued %d)",
                  h[1], h[2], h[3]);
    return fail(JXF_ERR_CUDA, "device error word 0x%x", h[0]);
  }
  return JXF_OK;
}

static __global__ void k_count_nonfinite(const float* f, long long n, int* count) {
  int local = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    local += !isfinite(f[i]);
  if (local) atomicAdd(count, local);
}

int jxf_grid3d_check_finite(jxf_grid3d* g, void* stream) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(cudaMemsetAsync(g->d_count, 0, 4, st));
  for (int k = 0; k < 6; ++k) k_count_nonfinite<<<592, 256, 0, st>>>(g->f[g->cur][k], g->n, g->d_count);
  CUDA_TRY(cudaGetLastError());
  int h = 0;
  CUDA_TRY(cudaMemcpyAsync(&h, g->d_count, 4, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (h) return fail(JXF_ERR_NONFINITE, "%d non-finite field values", h);
  return JXF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// 2D handle
// ---------------------------------------------------------------------------

struct jxf_grid2d {
  jxf_grid2d_desc d{};
  int mode = MODE_ABSORB;
  double dt = 0, coef_h = 0, coef_e = 0;
  long long n = 0;
  int64_t bytes = 0;
  float* f[3] = {};
  float* damp[2] = {};
  int n_src = 0;
  int* d_src_y = nullptr;
  float* d_src_amp = nullptr;
  int* d_src_wave = nullptr;
  std::vector<int> src_wave;
  float* d_wave = nullptr;
  int n_waves = 0;
  long long wave_len = 0;
  int n_wall = 0;
  int* d_wall_y = nullptr;
  int* d_wall_g0 = nullptr;
  int* d_wall_g1 = nullptr;
  long long step = 0;
};

extern "C" {

int jxf_grid2d_create(const jxf_grid2d_desc* desc, jxf_grid2d** out) {
  if (!desc || !out) return fail(JXF_ERR_INVALID, "null argument");
  *out = nullptr;
  const jxf_grid2d_desc d = *desc;
  if (d.nx < 3 || d.ny < 3) return fail(JXF_ERR_INVALID, "grid must be at least 3x3");
  if (!(d.dx > 0)) return fail(JXF_ERR_INVALID, "dx must be positive");
  if (d.pml_layers < 0) return fail(JXF_ERR_INVALID, "pml_layers must be >= 0");
  if (d.boundary != JXF_BND_ABSORBING && d.boundary != JXF_BND_PERIODIC &&
      d.boundary != JXF_BND_REFLECTING && d.boundary != JXF_BND_PEC)
    return fail(JXF_ERR_INVALID, "unsupported 2D boundary %d", d.boundary);
  DeviceGuard dg(d.device);
  if (!dg.ok) return fail(JXF_ERR_CUDA, "cannot select device %d", d.device);
  jxf_grid2d* g = new jxf_grid2d();
  g->d = d;
  g->n = (long long)d.nx * d.ny;
  g->dt = d.dt > 0 ? d.dt : 0.99 * d.dx / (kC0 * std::sqrt(2.0));  // fdtd.py:214
  g->coef_h = g->dt / (kMu0 * d.dx);                                // fdtd.py:254
  g->coef_e = g->dt / (kEps0 * d.dx);                               // fdtd.py:255
  g->mode = d.boundary == JXF_BND_PERIODIC     ? MODE_PERIODIC
            : d.boundary == JXF_BND_REFLECTING ? JXF_BND_REFLECTING
                                               : MODE_ABSORB;
  int rc;
  for (int k = 0; k < 3; ++k) {
    if ((rc = dmalloc(&g->f[k], (size_t)g->n, &g->bytes)) != JXF_OK) {
      jxf_grid2d_destroy(g);
      return rc;
    }
    cudaMemset(g->f[k], 0, (size_t)g->n * 4);
  }
  const int dims[2] = {d.nx, d.ny};
  for (int ax = 0; ax < 2; ++ax) {
    std::vector<float> t = d.boundary == JXF_BND_ABSORBING
                               ? damping_table(dims[ax], d.pml_layers, d.dx, g->dt, 2)
                               : std::vector<float>(dims[ax], 1.0f);
    if ((rc = upload(&g->damp[ax], t, &g->bytes)) != JXF_OK) {
      jxf_grid2d_destroy(g);
      return rc;
    }
  }
  cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    jxf_grid2d_destroy(g);
    return fail(JXF_ERR_CUDA, "initialisation failed: %s", cudaGetErrorString(e));
  }
  *out = g;
  return JXF_OK;
}

int jxf_grid2d_destroy(jxf_grid2d* g) {
  if (!g) return JXF_OK;
  DeviceGuard dg(g->d.device);
  for (int k = 0; k < 3; ++k) dfree(g->f[k]);
  for (int k = 0; k < 2; ++k) dfree(g->damp[k]);
  dfree(g->d_src_y);
  dfree(g->d_src_amp);
  dfree(g->d_src_wave);
  dfree(g->d_wave);
  dfree(g->d_wall_y);
  dfree(g->d_wall_g0);
  dfree(g->d_wall_g1);
  delete g;
  return JXF_OK;
}

int jxf_grid2d_set_sources(jxf_grid2d* g, int32_t n, const int32_t* y, const float* amplitude,
                           const int32_t* wave_id) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  if (n < 0 || (n > 0 && (!y || !amplitude || !wave_id)))
    return fail(JXF_ERR_INVALID, "bad source arrays");
  for (int i = 0; i < n; ++i) {
    if (y[i] < 0 || y[i] >= g->d.ny)
      return fail(JXF_ERR_INVALID, "source %d: y=%d out of grid bounds [0, %d)", i, y[i], g->d.ny);
    if (wave_id[i] < 0) return fail(JXF_ERR_INVALID, "source %d: negative wave id", i);
  }
  DeviceGuard dg(g->d.device);
  TRY(upload(&g->d_src_y, std::vector<int>(y, y + n), &g->bytes));
  TRY(upload(&g->d_src_amp, std::vector<float>(amplitude, amplitude + n), &g->bytes));
  TRY(upload(&g->d_src_wave, std::vector<int>(wave_id, wave_id + n), &g->bytes));
  g->src_wave.assign(wave_id, wave_id + n);
  g->n_src = n;
  return JXF_OK;
}

int jxf_grid2d_set_waveforms(jxf_grid2d* g, int32_t n_waves, int64_t n_samples,
                             const float* samples) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  if (n_waves < 0 || n_samples < 0 || (n_waves * n_samples > 0 && !samples))
    return fail(JXF_ERR_INVALID, "bad waveform table");
  DeviceGuard dg(g->d.device);
  TRY(upload(&g->d_wave, std::vector<float>(samples, samples + (size_t)n_waves * n_samples),
             &g->bytes));
  g->n_waves = n_waves;
  g->wave_len = n_samples;
  return JXF_OK;
}

int jxf_grid2d_set_walls(jxf_grid2d* g, int32_t n, const int32_t* y, const int32_t* gap_start,
                         const int32_t* gap_end) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  if (n < 0 || (n > 0 && (!y || !gap_start || !gap_end)))
    return fail(JXF_ERR_INVALID, "bad wall arrays");
  for (int i = 0; i < n; ++i)
    if (y[i] < 0 || y[i] >= g->d.ny)
      return fail(JXF_ERR_INVALID, "wall %d: y=%d out of grid bounds [0, %d)", i, y[i], g->d.ny);
  DeviceGuard dg(g->d.device);
  TRY(upload(&g->d_wall_y, std::vector<int>(y, y + n), &g->bytes));
  TRY(upload(&g->d_wall_g0, std::vector<int>(gap_start, gap_start + n), &g->bytes));
  TRY(upload(&g->d_wall_g1, std::vector<int>(gap_end, gap_end + n), &g->bytes));
  g->n_wall = n;
  return JXF_OK;
}

int jxf_grid2d_step(jxf_grid2d* g, int32_t n_steps, void* stream) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  if (n_steps < 0) return fail(JXF_ERR_INVALID, "n_steps must be >= 0");
  if (n_steps == 0) return JXF_OK;
  if (g->n_src > 0) {
    int max_w = 0;
    for (int w : g->src_wave) max_w = std::max(max_w, w);
    if (max_w >= g->n_waves)
      return fail(JXF_ERR_INVALID, "source wave id %d has no waveform row", max_w);
    if (g->step + n_steps > g->wave_len)
      return fail(JXF_ERR_INVALID, "waveform table covers %lld steps, need %lld", g->wave_len,
                  g->step + n_steps);
  }
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  Step2D p{};
  p.nx = g->d.nx;
  p.ny = g->d.ny;
  p.a = (float)g->coef_h;
  p.b = (float)g->coef_e;
  p.ez = g->f[0];
  p.hx = g->f[1];
  p.hy = g->f[2];
  p.damp[0] = g->damp[0];
  p.damp[1] = g->damp[1];
  p.n_src = g->n_src;
  p.src_y = g->d_src_y;
  p.src_amp = g->d_src_amp;
  p.src_wave = g->d_src_wave;
  p.wave = g->d_wave;
  p.wave_len = g->wave_len;
  p.n_wall = g->n_wall;
  p.wall_y = g->d_wall_y;
  p.wall_g0 = g->d_wall_g0;
  p.wall_g1 = g->d_wall_g1;
  const int threads = 256;
  const int blocks = (int)std::min<long long>((g->n + threads - 1) / threads, 148LL * 16);
  for (int k = 0; k < n_steps; ++k) {
    p.step = g->step;
    if (g->mode == MODE_PERIODIC) {
      k2d_h<MODE_PERIODIC><<<blocks, threads, 0, st>>>(p);
      k2d_e<MODE_PERIODIC, false><<<blocks, threads, 0, st>>>(p);
      k2d_post<MODE_PERIODIC><<<1, 1024, 0, st>>>(p);
    } else if (g->mode == JXF_BND_REFLECTING) {
      k2d_h<MODE_ABSORB><<<blocks, threads, 0, st>>>(p);
      k2d_e<MODE_PEC, false><<<blocks, threads, 0, st>>>(p);
      k2d_post<MODE_ABSORB><<<1, 1024, 0, st>>>(p);
    } else {
      k2d_h<MODE_ABSORB><<<blocks, threads, 0, st>>>(p);
      k2d_e<MODE_ABSORB, true><<<blocks, threads, 0, st>>>(p);
    }
    CUDA_TRY(cudaGetLastError());
    g->step++;
  }
  return JXF_OK;
}

int jxf_grid2d_reset(jxf_grid2d* g, void* stream) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  DeviceGuard dg(g->d.device);
  for (int k = 0; k < 3; ++k)
    CUDA_TRY(cudaMemsetAsync(g->f[k], 0, (size_t)g->n * 4, (cudaStream_t)stream));
  g->step = 0;
  return JXF_OK;
}

int jxf_grid2d_field_ptr(jxf_grid2d* g, int32_t comp, float** out) {
  if (!g || !out) return fail(JXF_ERR_INVALID, "null argument");
  if (comp < 0 || comp > 2) return fail(JXF_ERR_INVALID, "comp must be 0..2");
  *out = g->f[comp];
  return JXF_OK;
}

int jxf_grid2d_get_field(jxf_grid2d* g, int32_t comp, float* dst, int32_t dst_is_host,
                         void* stream) {
  if (!g || !dst) return fail(JXF_ERR_INVALID, "null argument");
  if (comp < 0 || comp > 2) return fail(JXF_ERR_INVALID, "comp must be 0..2");
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(cudaMemcpyAsync(dst, g->f[comp], (size_t)g->n * 4,
                           dst_is_host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice, st));
  if (dst_is_host) CUDA_TRY(cudaStreamSynchronize(st));
  return JXF_OK;
}

int jxf_grid2d_set_field(jxf_grid2d* g, int32_t comp, const float* src, int32_t src_is_host,
                         void* stream) {
  if (!g || !src) return fail(JXF_ERR_INVALID, "null argument");
  if (comp < 0 || comp > 2) return fail(JXF_ERR_INVALID, "comp must be 0..2");
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  CUDA_TRY(cudaMemcpyAsync(g->f[comp], src, (size_t)g->n * 4,
                           src_is_host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice, st));
  if (src_is_host) CUDA_TRY(cudaStreamSynchronize(st));
  return JXF_OK;
}

int jxf_grid2d_snapshot(jxf_grid2d* g, float* dst, void* stream) {
  if (!g || !dst) return fail(JXF_ERR_INVALID, "null argument");
  DeviceGuard dg(g->d.device);
  for (int k = 0; k < 3; ++k)
    CUDA_TRY(cudaMemcpyAsync(dst + (size_t)k * g->n, g->f[k], (size_t)g->n * 4,
                             cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return JXF_OK;
}

int jxf_grid2d_check_error(jxf_grid2d* g, void* stream) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  DeviceGuard dg(g->d.device);
  CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
  CUDA_TRY(cudaGetLastError());
  return JXF_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batches of independent grids
// ---------------------------------------------------------------------------

struct jxf_batch3d {
  std::vector<jxf_grid3d*> grids;
  int mode = MODE_ABSORB;
  int device = 0;
  int64_t bytes = 0;
  Step3D* d_params = nullptr;
  int* d_blk_grid = nullptr;
  int* d_blk_first = nullptr;
  int* d_blk_count = nullptr;
  int n_blocks = 0;
  BatchSrcGrid* d_srcg = nullptr;
  int2* d_src_entries = nullptr;
  int n_src_entries = 0;
  BatchProbe* d_probes = nullptr;
  int n_probes = 0;
  std::vector<int> probe_offset;  // first column of each grid in a probe row
  float* d_probe_buf = nullptr;   // [n_steps][n_probes] of the last run
  size_t probe_cap = 0;
  long long step = 0;
  cudaStream_t own = nullptr;     // capture stream when the caller passes the legacy stream
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaGraphExec_t graph = nullptr;
  long long graph_step0 = -1;
  int graph_n = -1;
  size_t cap[7] = {0, 0, 0, 0, 0, 0, 0};  // element capacity of the uploaded tables
  BandTables band;  // learned absorbing band (PEC batches only)
  // TMA batches (every member grid on the TMA path): one persistent launch
  // per step and CPML part over a work list of every grid's blocks
  bool tma = false;
  int cfg = -1, chunk = 0, axis_split = 0;
  bool cbarr = false, kappa = false, use_pdl = true;
  Step3D* d_tparams = nullptr;  // [2][n]: input set 0 / 1
  Maps3D* d_tmaps = nullptr;    // [2][n]
  int4* d_items = nullptr;      // parts concatenated
  int* d_counters = nullptr;    // [5][2]
  int part_off[5] = {0, 0, 0, 0, 0}, part_n[5] = {0, 0, 0, 0, 0}, part_ctas[5] = {0, 0, 0, 0, 0};
  size_t tcap[3] = {0, 0, 0};
  int graph_set = -1;           // input set at the start of the captured run
  bool tuned = false;
};

namespace {

// Dynamic shared-memory opt-in of a kernel, set once per kernel and device.
int tma_smem_optin(const void* k, size_t smem, int device) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> done;
  std::lock_guard<std::mutex> lk(mu);
  size_t& have = done[{k, device}];
  if (have < smem) {
    CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared));
    have = smem;
  }
  return JXF_OK;
}

// Persistent batch kernel and its shared memory for a part (0 shell, 1..3
// single-axis x / y / z shell, 4 interior; non-CPML batches use part 4).
void batch_tma_kernel(const jxf_batch3d* b, int part, TmaBatchKernel* k, size_t* smem) {
  const TmaConfig& c = tma_configs()[b->cfg];
  const int cb = b->cbarr ? 1 : 0;
  if (b->mode != MODE_CPML || part == 4) {
    *k = c.kb[0][cb];
    *smem = c.smem[0];
  } else if (part == 0) {
    *k = c.kb[b->kappa ? 2 : 1][cb];
    *smem = c.smem[1];
  } else {
    *k = c.kbax[part - 1][cb];
    *smem = c.smem_ax[part - 1];
  }
}

// One leapfrog step of a TMA batch: the parts' persistent launches chained by
// programmatic dependent launch (capturable).
int batch_tma_launch(jxf_batch3d* b, int in_set, long long step, cudaStream_t st) {
  const TmaConfig& c = tma_configs()[b->cfg];
  bool first = true;
  for (int pi = 0; pi < 5; ++pi) {
    if (b->part_n[pi] == 0) continue;
    TmaBatchKernel k;
    size_t smem;
    batch_tma_kernel(b, pi, &k, &smem);
    TmaBatchArgs a{};
    a.params = b->d_tparams;
    a.maps = b->d_tmaps;
    a.n_grids = (int)b->grids.size();
    a.in_set = in_set;
    a.items = b->d_items + b->part_off[pi];
    a.n_items = b->part_n[pi];
    a.counter = b->d_counters + 2 * pi;
    a.step = step;
    a.pdl = b->use_pdl ? (first ? (PDL_WAIT_START | PDL_TRIGGER) : (PDL_TRIGGER | PDL_WAIT_END))
                       : 0;
    cudaLaunchConfig_t lc{};
    lc.gridDim = dim3(b->part_ctas[pi], 1, 1);
    lc.blockDim = dim3(c.threads, 1, 1);
    lc.dynamicSmemBytes = smem;
    lc.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = b->use_pdl ? 1 : 0;
    lc.attrs = attr;
    lc.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&lc, k, a);
    if (e != cudaSuccess)
      return fail(JXF_ERR_CUDA, "batch step kernel launch failed: %s", cudaGetErrorString(e));
    first = false;
  }
  return JXF_OK;
}

// Launch tables of a TMA batch at its launch shape (b->cfg, b->chunk,
// b->axis_split): per-grid parameters and tensor maps for both input sets,
// per-block source lists, and the work items of every part (shell, x / y / z
// single-axis shell, interior for CPML; one part otherwise), each part's
// items heaviest first across all grids.  Buffers keep their addresses when
// large enough (a captured graph holds them); any reallocation drops the graph.
int batch_tma_tables(jxf_batch3d* b, bool* moved) {
  const int n = (int)b->grids.size();
  const TmaConfig& c = tma_configs()[b->cfg];
  std::vector<Step3D> params(2 * (size_t)n);
  std::vector<Maps3D> maps(2 * (size_t)n);
  struct Item {
    double cost;
    int4 w;
  };
  std::vector<Item> parts[5];
  const int warps = (c.threads + 31) / 32;
  for (int k = 0; k < n; ++k) {
    jxf_grid3d* g = b->grids[k];
    if (g->cfg != b->cfg || g->x_chunk != b->chunk) {
      g->cfg = b->cfg;
      g->x_chunk = b->chunk;
      g->maps_ok = false;
      g->built_cfg = -1;
    }
    g->axis_split = b->axis_split;
    g->tb = -1;
    if (!g->maps_ok || g->maps_cfg != g->cfg) TRY(encode_maps(g));
    if (!g->src_cell.empty() && (g->built_cfg != g->cfg || g->built_chunk != g->x_chunk))
      TRY(build_tma_sources(g));
    for (int s = 0; s < 2; ++s) {
      Step3D p = base_params(g);
      set_io(g, p, s, 1 - s);
      p.blk_src_ptr = g->src_cell.empty() ? nullptr : g->d_blk_ptr;
      p.src = g->d_entries;
      p.probe_out = nullptr;
      p.blk_list = nullptr;
      p.pdl = 0;
      p.x_chunk = b->chunk;
      p.ntiles_z = (g->d.nz + c.tz - 1) / c.tz;
      p.ntiles_y = (g->d.ny + c.ty - 1) / c.ty;
      params[(size_t)s * n + k] = p;
      maps[(size_t)s * n + k] = g->maps[s];
    }
    if (b->mode == MODE_CPML) {
      SplitLists sl;
      compute_split(g, b->cfg, b->chunk, b->axis_split != 0, sl);
      for (int pi = 0; pi < 5; ++pi)
        for (size_t i = 0; i < sl.cost[pi].size(); ++i)
          parts[pi].push_back({sl.cost[pi][i], make_int4(k, sl.list[pi][3 * i],
                                                         sl.list[pi][3 * i + 1],
                                                         sl.list[pi][3 * i + 2])});
    } else {
      const int ntz = (g->d.nz + c.tz - 1) / c.tz, nty = (g->d.ny + c.ty - 1) / c.ty;
      const int nch = (g->d.nx + b->chunk - 1) / b->chunk;
      for (int ch = 0; ch < nch; ++ch) {
        const int xb = ch * b->chunk, xe = std::min(xb + b->chunk, g->d.nx);
        const double cost = (double)(xe - std::max(xb - 1, 0)) * warps;
        for (int ty = 0; ty < nty; ++ty)
          for (int tz = 0; tz < ntz; ++tz) parts[4].push_back({cost, make_int4(k, tz, ty, ch)});
      }
    }
  }
  std::vector<int4> items;
  for (int pi = 0; pi < 5; ++pi) {
    std::stable_sort(parts[pi].begin(), parts[pi].end(),
                     [](const Item& u, const Item& v) { return u.cost > v.cost; });
    b->part_off[pi] = (int)items.size();
    b->part_n[pi] = (int)parts[pi].size();
    for (const Item& it : parts[pi]) items.push_back(it.w);
  }
  auto put = [&](auto** ptr, size_t* cap, const auto& v) -> int {
    if (v.empty()) return JXF_OK;
    if (*cap < v.size()) {
      dfree(*ptr);
      TRY(dmalloc(ptr, v.size(), &b->bytes));
      *cap = v.size();
      *moved = true;
    }
    CUDA_TRY(cudaMemcpy(*ptr, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice));
    return JXF_OK;
  };
  TRY(put(&b->d_tparams, &b->tcap[0], params));
  TRY(put(&b->d_tmaps, &b->tcap[1], maps));
  TRY(put(&b->d_items, &b->tcap[2], items));
  if (!b->d_counters) {
    TRY(dmalloc(&b->d_counters, 10, &b->bytes));
    CUDA_TRY(cudaMemset(b->d_counters, 0, 10 * sizeof(int)));
    *moved = true;
  }
  // persistent CTAs per part: resident blocks per SM times the SM count
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
  for (int pi = 0; pi < 5; ++pi) {
    b->part_ctas[pi] = 0;
    if (b->part_n[pi] == 0) continue;
    TmaBatchKernel k;
    size_t smem;
    batch_tma_kernel(b, pi, &k, &smem);
    TRY(tma_smem_optin(reinterpret_cast<const void*>(k), smem, b->device));
    int per_sm = 1;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, c.threads, smem));
    b->part_ctas[pi] = std::max(1, std::min(b->part_n[pi], std::max(per_sm, 1) * sms));
  }
  return JXF_OK;
}

int batch_refresh_tma(jxf_batch3d* b) {
  std::vector<BatchProbe> pr;
  b->probe_offset.clear();
  for (size_t k = 0; k < b->grids.size(); ++k) {
    jxf_grid3d* g = b->grids[k];
    b->probe_offset.push_back((int)pr.size());
    for (int i = 0; i < g->n_probes; ++i)
      pr.push_back(BatchProbe{(int)k, g->probe_comp_h[i], g->probe_cell_h[i]});
  }
  const int old_items = b->part_off[4] + b->part_n[4];
  int old_ctas[5];
  for (int i = 0; i < 5; ++i) old_ctas[i] = b->part_ctas[i];
  bool moved = false;
  TRY(batch_tma_tables(b, &moved));
  bool shape = b->n_probes != (int)pr.size() || old_items != b->part_off[4] + b->part_n[4];
  for (int i = 0; i < 5; ++i) shape = shape || old_ctas[i] != b->part_ctas[i];
  b->n_probes = (int)pr.size();
  if (!pr.empty() && b->cap[6] < pr.size()) {
    dfree(b->d_probes);
    TRY(dmalloc(&b->d_probes, pr.size(), &b->bytes));
    b->cap[6] = pr.size();
    moved = true;
  }
  if (!pr.empty())
    CUDA_TRY(cudaMemcpy(b->d_probes, pr.data(), pr.size() * sizeof(BatchProbe),
                        cudaMemcpyHostToDevice));
  if ((moved || shape) && b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return JXF_OK;
}

int batch_refresh(jxf_batch3d* b) {
  if (b->tma) return batch_refresh_tma(b);
  // parameters, block tables, sources and probes of every grid (cheap; done
  // per call so later set_eps / set_sources on the member grids are seen)
  std::vector<Step3D> params;
  std::vector<int> bg, bf, bc;
  std::vector<BatchSrcGrid> sg;
  std::vector<int2> se;
  std::vector<BatchProbe> pr;
  b->probe_offset.clear();
  int blocks = 0;
  for (size_t k = 0; k < b->grids.size(); ++k) {
    jxf_grid3d* g = b->grids[k];
    Step3D p = base_params(g);
    set_io(g, p, 0, 0);
    params.push_back(p);
    const long long cells = g->n;
    const int nb = (int)std::max<long long>(1, std::min<long long>((cells + 255) / 256, 4096));
    bf.push_back(blocks);
    bc.push_back(nb);
    for (int i = 0; i < nb; ++i) bg.push_back((int)k);
    blocks += nb;
    BatchSrcGrid s{};
    for (int c = 0; c < 3; ++c) s.e[c] = g->f[0][c];
    s.cells = g->d_cells;
    s.terms = g->d_terms;
    s.wave = g->d_wave;
    s.wave_len = g->wave_len;
    sg.push_back(s);
    for (int i = 0; i < g->n_cells; ++i) se.push_back(make_int2((int)k, i));
    b->probe_offset.push_back((int)pr.size());
    if (g->n_probes > 0) {
      std::vector<long long> cell(g->n_probes);
      std::vector<int> comp(g->n_probes);
      CUDA_TRY(cudaMemcpy(cell.data(), g->d_probe_cell, cell.size() * 8, cudaMemcpyDeviceToHost));
      CUDA_TRY(cudaMemcpy(comp.data(), g->d_probe_comp, comp.size() * 4, cudaMemcpyDeviceToHost));
      for (int i = 0; i < g->n_probes; ++i) pr.push_back(BatchProbe{(int)k, comp[i], cell[i]});
    }
  }
  if (b->n_blocks != blocks || b->n_src_entries != (int)se.size() ||
      b->n_probes != (int)pr.size()) {
    // launch shapes are part of a captured graph
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  b->n_blocks = blocks;
  b->n_src_entries = (int)se.size();
  b->n_probes = (int)pr.size();
  // Copy into the existing buffers when they are large enough: a captured
  // graph keeps these device addresses.  Any reallocation drops the graph.
  bool moved = false;
  auto put = [&](auto** ptr, size_t* cap, const auto& v) -> int {
    if (v.empty()) return JXF_OK;
    if (*cap < v.size()) {
      dfree(*ptr);
      TRY(dmalloc(ptr, v.size(), &b->bytes));
      *cap = v.size();
      moved = true;
    }
    CUDA_TRY(cudaMemcpy(*ptr, v.data(), v.size() * sizeof(v[0]), cudaMemcpyHostToDevice));
    return JXF_OK;
  };
  TRY(put(&b->d_params, &b->cap[0], params));
  TRY(put(&b->d_blk_grid, &b->cap[1], bg));
  TRY(put(&b->d_blk_first, &b->cap[2], bf));
  TRY(put(&b->d_blk_count, &b->cap[3], bc));
  TRY(put(&b->d_srcg, &b->cap[4], sg));
  TRY(put(&b->d_src_entries, &b->cap[5], se));
  TRY(put(&b->d_probes, &b->cap[6], pr));
  if (moved && b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return JXF_OK;
}

// One leapfrog step of every grid (kernels only; capturable).  TMA batches
// read buffer set `in_set` and write the other one.
int batch_launch_step(jxf_batch3d* b, long long step, float* probe_row, cudaStream_t st,
                      int in_set = 0) {
  if (b->tma) {
    TRY(batch_tma_launch(b, in_set, step, st));
    if (b->band.band) TRY(band_launch(b->band, st, in_set ^ 1));
    if (probe_row && b->n_probes > 0)
      k3d_batch_probes<<<(b->n_probes + 127) / 128, 128, 0, st>>>(
          b->d_tparams + (size_t)(in_set ^ 1) * b->grids.size(), b->d_probes, b->n_probes,
          probe_row);
    CUDA_TRY(cudaGetLastError());
    return JXF_OK;
  }
  BatchBlocks bb{b->d_params, b->d_blk_grid, b->d_blk_first, b->d_blk_count};
  if (b->mode == MODE_CPML) {
    k3d_batch_h<MODE_CPML><<<b->n_blocks, 256, 0, st>>>(bb);
    k3d_batch_e<MODE_CPML><<<b->n_blocks, 256, 0, st>>>(bb);
  } else {
    k3d_batch_h<MODE_ABSORB><<<b->n_blocks, 256, 0, st>>>(bb);
    k3d_batch_e<MODE_ABSORB><<<b->n_blocks, 256, 0, st>>>(bb);
  }
  if (b->n_src_entries > 0)
    k3d_batch_sources<<<(b->n_src_entries + 127) / 128, 128, 0, st>>>(b->d_srcg, b->d_src_entries,
                                                                      b->n_src_entries, step);
  if (b->band.band) TRY(band_launch(b->band, st));
  if (probe_row && b->n_probes > 0)
    k3d_batch_probes<<<(b->n_probes + 127) / 128, 128, 0, st>>>(b->d_params, b->d_probes,
                                                                b->n_probes, probe_row);
  CUDA_TRY(cudaGetLastError());
  return JXF_OK;
}

}  // namespace

namespace {

// Launch shape of a TMA batch: every registry shape offered for batches x
// chunk {4, 8, 16} x single-axis split (CPML, kappa = 1), each timed over two
// steps into the idle buffer sets (the state is untouched), best of two
// trials.  JXF_BATCH_LAUNCH=cfg,chunk[,split] pins it.
int batch_tma_tune(jxf_batch3d* b, int in_set, cudaStream_t st) {
  b->tuned = true;
  const char* forced = std::getenv("JXF_BATCH_LAUNCH");
  int fc = -1, fk = -1, fs = 0;
  if (forced && std::sscanf(forced, "%d,%d,%d", &fc, &fk, &fs) >= 2 && fc >= 0 &&
      fc < (int)tma_configs().size() && tma_configs()[fc].kb[0][0] && fk >= 1) {
    b->cfg = fc;
    b->chunk = fk;
    b->axis_split = fs != 0 ? 1 : 0;
    return JXF_OK;
  }
  const char* env = std::getenv("JXF_AUTOTUNE");
  if (env && env[0] == '0') return JXF_OK;
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  float best = 1e30f;
  int bc = b->cfg, bk = b->chunk, bs = b->axis_split;
  const bool can_split = b->mode == MODE_CPML && !b->kappa;
  for (int sp = 0; sp < (can_split ? 2 : 1); ++sp)
    for (int ci = 0; ci < (int)tma_configs().size(); ++ci) {
      if (!tma_configs()[ci].kb[0][0]) continue;
      for (int ch : {4, 8, 16}) {
        b->cfg = ci;
        b->chunk = ch;
        b->axis_split = sp;
        bool moved = false;
        TRY(batch_tma_tables(b, &moved));
        TRY(batch_tma_launch(b, in_set, b->step, st));
        float ms = 1e30f;
        for (int trial = 0; trial < 2; ++trial) {
          CUDA_TRY(cudaEventRecord(e0, st));
          for (int r = 0; r < 2; ++r) TRY(batch_tma_launch(b, in_set, b->step, st));
          CUDA_TRY(cudaEventRecord(e1, st));
          CUDA_TRY(cudaEventSynchronize(e1));
          float t = 0;
          CUDA_TRY(cudaEventElapsedTime(&t, e0, e1));
          ms = std::min(ms, t);
        }
        if (ms < best) {
          best = ms;
          bc = ci;
          bk = ch;
          bs = sp;
        }
      }
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  b->cfg = bc;
  b->chunk = bk;
  b->axis_split = bs;
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  return JXF_OK;
}

}  // namespace

extern "C" int jxf_batch3d_create(int32_t n, jxf_grid3d* const* grids, jxf_batch3d** out) {
  if (!out || n < 1 || !grids) return fail(JXF_ERR_INVALID, "need at least one grid");
  *out = nullptr;
  if (!grids[0]) return fail(JXF_ERR_INVALID, "grid 0 is null");
  const int mode = grids[0]->mode;
  const int dev = grids[0]->d.device;
  const int path = grids[0]->path;
  for (int i = 0; i < n; ++i) {
    const jxf_grid3d* g = grids[i];
    if (!g) return fail(JXF_ERR_INVALID, "grid %d is null", i);
    if (g->slab) return fail(JXF_ERR_INVALID, "grid %d: x-slab grids are not batched", i);
    if (g->path != path)
      return fail(JXF_ERR_INVALID, "grid %d: batched grids share the kernel path", i);
    if (g->mode != mode || g->d.device != dev)
      return fail(JXF_ERR_INVALID, "grid %d: batched grids share the boundary mode and device", i);
    if (g->mode == MODE_PERIODIC) return fail(JXF_ERR_INVALID, "periodic grids are not batched");
    if (path == JXF_PATH_TMA) {
      if ((g->cb != nullptr) != (grids[0]->cb != nullptr))
        return fail(JXF_ERR_INVALID,
                    "grid %d: TMA batches need a permittivity map on every grid or on none", i);
      if (g->kappa != grids[0]->kappa)
        return fail(JXF_ERR_INVALID, "grid %d: TMA batches share the CPML kappa grading", i);
    }
  }
  DeviceGuard dg(dev);
  jxf_batch3d* b = new jxf_batch3d();
  b->grids.assign(grids, grids + n);
  b->mode = mode;
  b->device = dev;
  b->tma = path == JXF_PATH_TMA;
  b->cbarr = grids[0]->cb != nullptr;
  b->kappa = grids[0]->kappa;
  {
    const char* e = std::getenv("JXF_PDL");
    b->use_pdl = !(e && e[0] == '0');
  }
  if (b->tma) {
    // a first launch shape; jxf_batch3d_step tunes it on the first run
    b->cfg = 0;
    b->chunk = 8;
    b->axis_split = 0;
  }
  int rc = batch_refresh(b);
  if (rc != JXF_OK) {
    jxf_batch3d_destroy(b);
    return rc;
  }
  *out = b;
  return JXF_OK;
}

extern "C" int jxf_batch3d_destroy(jxf_batch3d* b) {
  if (!b) return JXF_OK;
  DeviceGuard dg(b->device);
  if (b->graph) cudaGraphExecDestroy(b->graph);
  if (b->own) cudaStreamDestroy(b->own);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  dfree(b->d_params);
  dfree(b->d_blk_grid);
  dfree(b->d_blk_first);
  dfree(b->d_blk_count);
  dfree(b->d_srcg);
  dfree(b->d_src_entries);
  dfree(b->d_probes);
  dfree(b->d_probe_buf);
  dfree(b->d_tparams);
  dfree(b->d_tmaps);
  dfree(b->d_items);
  dfree(b->d_counters);
  band_release(b->band);
  delete b;
  return JXF_OK;
}

extern "C" int jxf_batch3d_reset(jxf_batch3d* b, void* stream) {
  if (!b) return fail(JXF_ERR_INVALID, "null handle");
  for (jxf_grid3d* g : b->grids) TRY(jxf_grid3d_reset(g, stream));
  b->step = 0;
  return JXF_OK;
}

extern "C" int jxf_batch3d_step(jxf_batch3d* b, int32_t n_steps, int32_t use_graph, void* stream) {
  if (!b) return fail(JXF_ERR_INVALID, "null handle");
  if (n_steps < 0) return fail(JXF_ERR_INVALID, "n_steps must be >= 0");
  if (n_steps == 0) return JXF_OK;
  for (jxf_grid3d* g : b->grids) {
    if (!g->src_cell.empty() && b->step + n_steps > g->wave_len)
      return fail(JXF_ERR_INVALID, "a member grid's waveform table is too short");
  }
  DeviceGuard dg(b->device);
  int in_set = 0;
  if (b->tma) {
    in_set = b->grids[0]->cur;
    for (jxf_grid3d* g : b->grids)
      if (g->cur != in_set)
        return fail(JXF_ERR_INVALID,
                    "TMA batch members must hold their state in the same buffer set (step "
                    "parity); reset the batch or step the grids to equal parity");
    if (!b->tuned) TRY(batch_tma_tune(b, in_set, (cudaStream_t)stream));
  }
  TRY(batch_refresh(b));
  const size_t need = (size_t)n_steps * std::max(b->n_probes, 1);
  if (need > b->probe_cap) {
    dfree(b->d_probe_buf);
    TRY(dmalloc(&b->d_probe_buf, need, &b->bytes));
    b->probe_cap = need;
    if (b->graph) {
      cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
    }
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (!use_graph) {
    for (int k = 0; k < n_steps; ++k)
      TRY(batch_launch_step(b, b->step + k,
                            b->n_probes ? b->d_probe_buf + (size_t)k * b->n_probes : nullptr, st,
                            in_set ^ (k & 1)));
  } else {
    if (!b->own) {
      CUDA_TRY(cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking));
      CUDA_TRY(cudaEventCreateWithFlags(&b->ev0, cudaEventDisableTiming));
      CUDA_TRY(cudaEventCreateWithFlags(&b->ev1, cudaEventDisableTiming));
    }
    if (!b->graph || b->graph_n != n_steps || b->graph_step0 != b->step ||
        b->graph_set != in_set) {
      if (b->graph) cudaGraphExecDestroy(b->graph);
      b->graph = nullptr;
      cudaGraph_t graph;
      CUDA_TRY(cudaStreamBeginCapture(b->own, cudaStreamCaptureModeThreadLocal));
      for (int k = 0; k < n_steps; ++k) {
        int rc = batch_launch_step(
            b, b->step + k, b->n_probes ? b->d_probe_buf + (size_t)k * b->n_probes : nullptr,
            b->own, in_set ^ (k & 1));
        if (rc != JXF_OK) {
          cudaStreamEndCapture(b->own, &graph);
          return rc;
        }
      }
      CUDA_TRY(cudaStreamEndCapture(b->own, &graph));
      CUDA_TRY(cudaGraphInstantiate(&b->graph, graph, 0));
      cudaGraphDestroy(graph);
      b->graph_n = n_steps;
      b->graph_step0 = b->step;
      b->graph_set = in_set;
    }
    // order the graph between the caller's earlier and later work
    CUDA_TRY(cudaEventRecord(b->ev0, st));
    CUDA_TRY(cudaStreamWaitEvent(b->own, b->ev0, 0));
    CUDA_TRY(cudaGraphLaunch(b->graph, b->own));
    CUDA_TRY(cudaEventRecord(b->ev1, b->own));
    CUDA_TRY(cudaStreamWaitEvent(st, b->ev1, 0));
  }
  b->step += n_steps;
  for (jxf_grid3d* g : b->grids) {
    g->step += n_steps;
    if (b->tma) g->cur ^= (n_steps & 1);
  }
  return JXF_OK;
}

extern "C" int jxf_batch3d_kernels_per_step(const jxf_batch3d* b) {
  if (!b) return 0;
  int n = 0;
  if (b->tma) {
    for (int i = 0; i < 5; ++i) n += b->part_n[i] > 0 ? 1 : 0;
  } else {
    n = 2 + (b->n_src_entries > 0 ? 1 : 0);
  }
  if (b->band.band) n += 2;
  if (b->n_probes > 0) n += 1;
  return n;
}

extern "C" int jxf_batch3d_launch(const jxf_batch3d* b, int32_t* out3) {
  if (!b || !out3) return fail(JXF_ERR_INVALID, "null argument");
  out3[0] = b->tma ? b->cfg : -1;
  out3[1] = b->tma ? b->chunk : -1;
  out3[2] = b->tma ? b->axis_split : -1;
  return JXF_OK;
}

extern "C" int jxf_batch3d_probes(jxf_batch3d* b, int32_t grid, int32_t n_steps, float* dst,
                                  void* stream) {
  if (!b || !dst) return fail(JXF_ERR_INVALID, "null argument");
  if (grid < 0 || grid >= (int)b->grids.size()) return fail(JXF_ERR_INVALID, "grid out of range");
  const int np = b->grids[grid]->n_probes;
  if (np == 0) return JXF_OK;
  if ((size_t)n_steps * b->n_probes > b->probe_cap)
    return fail(JXF_ERR_INVALID, "no probe rows for %d steps", n_steps);
  DeviceGuard dg(b->device);
  CUDA_TRY(cudaMemcpy2DAsync(dst, np * 4, b->d_probe_buf + b->probe_offset[grid],
                             (size_t)b->n_probes * 4, np * 4, n_steps, cudaMemcpyDeviceToDevice,
                             (cudaStream_t)stream));
  return JXF_OK;
}

// ---------------------------------------------------------------------------
// Learned absorbing band
// ---------------------------------------------------------------------------

struct jxf_band {
  int device = 0;
  int64_t bytes = 0;
  float* d_params = nullptr;  // [6][kParams] FP32 master
  float* d_grad = nullptr;
  float* d_m1 = nullptr;
  float* d_m2 = nullptr;
  unsigned char* d_wimg = nullptr;  // [6][kImgBytes] BF16 operand images
  float* d_loss = nullptr;          // [loss_cap][6]
  size_t loss_cap = 0;
  double* d_wsum = nullptr;         // [6] sum of row weights
  int* d_err = nullptr;
  long long adam_t = 0;
  // training rows per face
  __nv_bfloat16* feat[6] = {};
  float* tgt[6] = {};
  float* w[6] = {};
  long long rows[6] = {};
  long long cap[6] = {};
  int* d_cells = nullptr;  // collect scratch
  size_t cells_cap = 0;
  int attached = 0;        // grids and batches applying this band
};

namespace {

int band_setup_attrs() {
  static int done = 0;
  if (!done) {
    CUDA_TRY(cudaFuncSetAttribute(band::k_band_infer<band::SRC_GRIDS>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, band::kInfSmem));
    CUDA_TRY(cudaFuncSetAttribute(band::k_band_infer<band::SRC_ROWS>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, band::kInfSmem));
    CUDA_TRY(cudaFuncSetAttribute(band::k_band_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  band::kTrSmem));
    // The carveout is only a hint, and without one the driver may configure
    // less shared memory than the CTAs per SM the grid is sized for (the
    // launch then runs in several waves): ask for the largest split.
    CUDA_TRY(cudaFuncSetAttribute(band::k_band_infer<band::SRC_GRIDS>,
                                  cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared));
    CUDA_TRY(cudaFuncSetAttribute(band::k_band_infer<band::SRC_ROWS>,
                                  cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared));
    CUDA_TRY(cudaFuncSetAttribute(band::k_band_train, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared));
    done = 1;
  }
  return JXF_OK;
}

// Owning face of an outer-layer cell, or -1 for an inner cell.
int band_owner(int x, int y, int z, int nx, int ny, int nz) {
  const int c[3] = {x, y, z}, n[3] = {nx, ny, nz};
  int ax[3], sd[3], k = 0;
  for (int a = 0; a < 3; ++a) {
    if (c[a] == 0) {
      ax[k] = a;
      sd[k++] = 0;
    } else if (c[a] == n[a] - 1) {
      ax[k] = a;
      sd[k++] = 1;
    }
  }
  if (k == 0) return -1;
  if (k == 1 || k == 3) return 2 * ax[0] + sd[0];
  const int a = ax[0], b = ax[1];
  return (b == (a + 1) % 3) ? 2 * a + sd[0] : 2 * b + sd[1];
}

// Outer-layer cells of an nx*ny*nz grid, per owning face: x and y faces in
// ascending cell order (neighbouring lanes read neighbouring z), z faces in
// (y, x) order (neighbouring lanes step along x, the stencil's tangent axis,
// so they share the stencil rows x-1, x, x+1).
void band_cells(int nx, int ny, int nz, std::vector<int> out[6]) {
  for (int f = 0; f < 6; ++f) out[f].clear();
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y) {
      const bool full = x == 0 || x == nx - 1 || y == 0 || y == ny - 1;
      for (int z = 0; z < nz; z += (full || z == nz - 1) ? 1 : nz - 1) {
        const int f = band_owner(x, y, z, nx, ny, nz);
        if (f >= 0) out[f].push_back((x * ny + y) * nz + z);
      }
    }
  for (int f = 4; f < 6; ++f)
    std::stable_sort(out[f].begin(), out[f].end(), [&](int a, int b) {
      const int ya = (a / nz) % ny, yb = (b / nz) % ny;
      return ya != yb ? ya < yb : a < b;
    });
}

int band_check_dims(int nx, int ny, int nz) {
  if (nx < 8 || ny < 8 || nz < 8)
    return fail(JXF_ERR_INVALID, "a learned band needs every grid side >= 8 (got %d x %d x %d)",
                nx, ny, nz);
  if ((long long)nx * ny * nz >= (1ll << 31))
    return fail(JXF_ERR_INVALID, "a learned band grid must have fewer than 2^31 cells");
  return JXF_OK;
}

// Band correction of the state held in buffer set `set` of every grid.
int band_launch(const BandTables& t, cudaStream_t st, int set) {
  if (t.tiles <= 0) return JXF_OK;
  const band::GridRef* grids = (set != 0 && t.d_grids_b) ? t.d_grids_b : t.d_grids;
  band::InferArgs a{};
  a.grids = grids;
  a.cells = t.d_cells;
  a.tile_face = t.d_tile_face;
  a.n_tiles = t.tiles;
  a.wimg = t.band->d_wimg;
  a.params = t.band->d_params;
  a.delta = t.d_delta;
  a.err = t.band->d_err;
  a.wait_ns = wait_limit_ns();
  {
    // fault injection for tests (read at every launch): JXF_FAULT_DROP_MMA=1
    const char* e = std::getenv("JXF_FAULT_DROP_MMA");
    a.drop_first_mma = (e && e[0] == '1') ? 1 : 0;
  }
  band::k_band_infer<band::SRC_GRIDS><<<t.ctas, 128, band::kInfSmem, st>>>(a);
  const int n = t.tiles * band::kTile;
  band::k_band_apply<<<(n + 255) / 256, 256, 0, st>>>(grids, t.d_cells, n, t.d_delta,
                                                      t.band->d_err);
  CUDA_TRY(cudaGetLastError());
  return JXF_OK;
}

void band_release(BandTables& t) {
  if (t.band) t.band->attached -= 1;
  dfree(t.d_grids);
  dfree(t.d_grids_b);
  dfree(t.d_cells);
  dfree(t.d_tile_face);
  dfree(t.d_delta);
  t.band = nullptr;
  t.tiles = 0;
}

// CTAs of the inference kernel: resident CTAs per SM (limited by shared
// memory, registers and the SM's 512 TMEM columns) times the SM count.
int band_ctas(int n_tiles, int device) {
  int sms = 148, smem_sm = 233472, regs_sm = 65536;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device);
  cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, device);
  cudaFuncAttributes fa{};
  int regs = 128;
  if (cudaFuncGetAttributes(&fa, band::k_band_infer<band::SRC_GRIDS>) == cudaSuccess)
    regs = std::max(fa.numRegs, 1);
  cudaGetLastError();
  const int by_smem = smem_sm / (band::kInfSmem + 1024);
  const int by_regs = regs_sm / (regs * 128);
  const int by_tmem = 512 / band::kInfTmemCols;
  // (the runtime's occupancy query reports 1 block per SM for this kernel,
  // while 5 run side by side: measured, so the count comes from the limits)
  const int occ = std::max(1, std::min(std::min(by_smem, by_regs), by_tmem));
  return std::max(1, std::min(n_tiles, sms * occ));
}

// Face lists -> padded tile arrays.
void band_tiles(const std::vector<int2> per_face[6], std::vector<int2>& cells,
                std::vector<int>& tile_face) {
  cells.clear();
  tile_face.clear();
  for (int f = 0; f < 6; ++f) {
    const size_t n = per_face[f].size();
    const size_t nt = (n + band::kTile - 1) / band::kTile;
    for (size_t t = 0; t < nt; ++t) tile_face.push_back(f);
    for (size_t i = 0; i < nt * band::kTile; ++i)
      cells.push_back(i < n ? per_face[f][i] : make_int2(-1, 0));
  }
}

int band_grow(jxf_band* m, int f, long long need) {
  if (need <= m->cap[f]) return JXF_OK;
  long long nc = std::max<long long>(need, std::max<long long>(65536, m->cap[f] * 2));
  __nv_bfloat16* nf = nullptr;
  float *nt = nullptr, *nw = nullptr;
  TRY(dmalloc(&nf, (size_t)nc * band::kInP, &m->bytes));
  TRY(dmalloc(&nt, (size_t)nc * band::kOut, &m->bytes));
  TRY(dmalloc(&nw, (size_t)nc, &m->bytes));
  if (m->rows[f] > 0) {
    CUDA_TRY(cudaMemcpy(nf, m->feat[f], (size_t)m->rows[f] * band::kInP * 2,
                        cudaMemcpyDeviceToDevice));
    CUDA_TRY(cudaMemcpy(nt, m->tgt[f], (size_t)m->rows[f] * band::kOut * 4,
                        cudaMemcpyDeviceToDevice));
    CUDA_TRY(cudaMemcpy(nw, m->w[f], (size_t)m->rows[f] * 4, cudaMemcpyDeviceToDevice));
  }
  m->bytes -= (int64_t)m->cap[f] * (band::kInP * 2 + band::kOut * 4 + 4);
  dfree(m->feat[f]);
  dfree(m->tgt[f]);
  dfree(m->w[f]);
  m->feat[f] = nf;
  m->tgt[f] = nt;
  m->w[f] = nw;
  m->cap[f] = nc;
  return JXF_OK;
}

__global__ void k_band_wsum(const float* w, long long n, double* out) {
  double s = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    s += w[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

int band_weight_sums(jxf_band* m, double out[6], cudaStream_t st) {
  CUDA_TRY(cudaMemsetAsync(m->d_wsum, 0, 6 * sizeof(double), st));
  for (int f = 0; f < 6; ++f)
    if (m->rows[f] > 0)
      k_band_wsum<<<256, 256, 0, st>>>(m->w[f], m->rows[f], m->d_wsum + f);
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaMemcpyAsync(out, m->d_wsum, 6 * sizeof(double), cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return JXF_OK;
}

int band_pack(jxf_band* m, cudaStream_t st) {
  band::k_band_pack<<<dim3((band::kImgBytes / 2 + 255) / 256, 6), 256, 0, st>>>(m->d_params,
                                                                                m->d_wimg);
  CUDA_TRY(cudaGetLastError());
  return JXF_OK;
}

int band_train_pass(jxf_band* m, const band::TrainArgs& a, cudaStream_t st) {
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, m->device);
  int maxt = 0;
  for (int f = 0; f < 6; ++f) maxt = std::max(maxt, a.tiles[f]);
  if (maxt == 0) return JXF_OK;
  const int gx = std::max(1, std::min(maxt, std::max(1, sms / 6)));
  band::k_band_train<<<dim3(gx, 6), 128, band::kTrSmem, st>>>(a);
  CUDA_TRY(cudaGetLastError());
  return JXF_OK;
}

// Tables for the outer cells of `grids` (PEC, sides >= 8).
int band_attach(const std::vector<jxf_grid3d*>& grids, jxf_band* m, int device, int64_t* tally,
                BandTables& t) {
  if (m->device != device) return fail(JXF_ERR_INVALID, "band and grids on different devices");
  std::vector<band::GridRef> refs, refs_b;
  std::vector<int2> per[6];
  std::vector<int> cells[6];
  for (size_t k = 0; k < grids.size(); ++k) {
    jxf_grid3d* g = grids[k];
    if (g->d.boundary != JXF_BND_PEC)
      return fail(JXF_ERR_INVALID, "grid %zu: a learned band needs PEC-walled grids", k);
    TRY(band_check_dims(g->d.nx, g->d.ny, g->d.nz));
    band::GridRef r{};
    for (int c = 0; c < 6; ++c) r.f[c] = g->f[0][c];
    r.nx = g->d.nx;
    r.ny = g->d.ny;
    r.nz = g->d.nz;
    refs.push_back(r);
    for (int c = 0; c < 6; ++c) r.f[c] = g->f[1][c];
    refs_b.push_back(r);
    band_cells(g->d.nx, g->d.ny, g->d.nz, cells);
    for (int f = 0; f < 6; ++f)
      for (int c : cells[f]) per[f].push_back(make_int2(c, (int)k));
  }
  std::vector<int2> tc;
  std::vector<int> tf;
  band_tiles(per, tc, tf);
  BandTables n{};
  int rc = upload(&n.d_grids, refs, tally);
  if (rc == JXF_OK) rc = upload(&n.d_grids_b, refs_b, tally);
  if (rc == JXF_OK) rc = upload(&n.d_cells, tc, tally);
  if (rc == JXF_OK) rc = upload(&n.d_tile_face, tf, tally);
  if (rc == JXF_OK) rc = dmalloc(&n.d_delta, tc.size() * band::kOut, tally);
  if (rc != JXF_OK) {
    band_release(n);
    return rc;
  }
  n.tiles = (int)tf.size();
  n.ctas = band_ctas(n.tiles, device);
  n.band = m;
  m->attached += 1;
  t = n;
  return JXF_OK;
}

band::TrainArgs band_train_args(jxf_band* m) {
  band::TrainArgs a{};
  for (int f = 0; f < 6; ++f) {
    a.feat[f] = m->feat[f];
    a.tgt[f] = m->tgt[f];
    a.w[f] = m->w[f];
    a.count[f] = m->rows[f];
  }
  a.wimg = m->d_wimg;
  a.params = m->d_params;
  a.grad = m->d_grad;
  a.err = m->d_err;
  a.wait_ns = wait_limit_ns();
  return a;
}

}  // namespace

extern "C" {

int jxf_band_create(int32_t device, jxf_band** out) {
  if (!out) return fail(JXF_ERR_INVALID, "null output");
  *out = nullptr;
  int ndev = 0;
  CUDA_TRY(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(JXF_ERR_INVALID, "device %d out of range", device);
  DeviceGuard dg(device);
  TRY(band_setup_attrs());
  jxf_band* m = new jxf_band();
  m->device = device;
  const size_t np = 6 * (size_t)band::kParams;
  int rc = JXF_OK;
  if (rc == JXF_OK) rc = dmalloc(&m->d_params, np, &m->bytes);
  if (rc == JXF_OK) rc = dmalloc(&m->d_grad, np, &m->bytes);
  if (rc == JXF_OK) rc = dmalloc(&m->d_m1, np, &m->bytes);
  if (rc == JXF_OK) rc = dmalloc(&m->d_m2, np, &m->bytes);
  if (rc == JXF_OK) rc = dmalloc(&m->d_wimg, 6 * (size_t)band::kImgBytes, &m->bytes);
  if (rc == JXF_OK) rc = dmalloc(&m->d_wsum, 6, &m->bytes);
  if (rc == JXF_OK) rc = dmalloc(&m->d_err, 4, &m->bytes);
  if (rc == JXF_OK && cudaMemset(m->d_params, 0, np * 4) != cudaSuccess) rc = JXF_ERR_CUDA;
  if (rc == JXF_OK && cudaMemset(m->d_m1, 0, np * 4) != cudaSuccess) rc = JXF_ERR_CUDA;
  if (rc == JXF_OK && cudaMemset(m->d_m2, 0, np * 4) != cudaSuccess) rc = JXF_ERR_CUDA;
  if (rc == JXF_OK && cudaMemset(m->d_err, 0, 16) != cudaSuccess) rc = JXF_ERR_CUDA;
  if (rc == JXF_OK) rc = band_pack(m, 0);
  if (rc == JXF_OK && cudaDeviceSynchronize() != cudaSuccess) rc = JXF_ERR_CUDA;
  if (rc != JXF_OK) {
    jxf_band_destroy(m);
    return rc == JXF_ERR_CUDA ? fail(rc, "band allocation failed") : rc;
  }
  *out = m;
  return JXF_OK;
}

int jxf_band_destroy(jxf_band* m) {
  if (!m) return JXF_OK;
  if (m->attached > 0)
    return fail(JXF_ERR_INVALID, "the band is still attached to %d grid(s) or batch(es)",
                m->attached);
  DeviceGuard dg(m->device);
  cudaDeviceSynchronize();
  dfree(m->d_params);
  dfree(m->d_grad);
  dfree(m->d_m1);
  dfree(m->d_m2);
  dfree(m->d_wimg);
  dfree(m->d_loss);
  dfree(m->d_wsum);
  dfree(m->d_err);
  dfree(m->d_cells);
  for (int f = 0; f < 6; ++f) {
    dfree(m->feat[f]);
    dfree(m->tgt[f]);
    dfree(m->w[f]);
  }
  delete m;
  return JXF_OK;
}

int jxf_band_set_params(jxf_band* m, const float* params) {
  if (!m || !params) return fail(JXF_ERR_INVALID, "null argument");
  DeviceGuard dg(m->device);
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpy(m->d_params, params, 6 * (size_t)band::kParams * 4, cudaMemcpyHostToDevice));
  // padding entries are zero by definition (an Adam pass with lr = 0 and a zero gradient)
  CUDA_TRY(cudaMemset(m->d_grad, 0, 6 * (size_t)band::kParams * 4));
  band::k_band_adam<<<(6 * band::kParams + 255) / 256, 256>>>(
      m->d_params, m->d_grad, m->d_m1, m->d_m2, 6 * band::kParams, 0.0f, 0.9f, 0.999f, 1e-8f,
      1.0f, 1.0f);
  CUDA_TRY(cudaMemset(m->d_m1, 0, 6 * (size_t)band::kParams * 4));
  CUDA_TRY(cudaMemset(m->d_m2, 0, 6 * (size_t)band::kParams * 4));
  m->adam_t = 0;
  TRY(band_pack(m, 0));
  CUDA_TRY(cudaDeviceSynchronize());
  return JXF_OK;
}

int jxf_band_get_params(jxf_band* m, float* params) {
  if (!m || !params) return fail(JXF_ERR_INVALID, "null argument");
  DeviceGuard dg(m->device);
  CUDA_TRY(cudaDeviceSynchronize());
  CUDA_TRY(cudaMemcpy(params, m->d_params, 6 * (size_t)band::kParams * 4, cudaMemcpyDeviceToHost));
  return JXF_OK;
}

int jxf_band_eval(jxf_band* m, int32_t n, const float* feat, const int32_t* face, float* out) {
  if (!m || n < 0 || (n > 0 && (!feat || !face || !out)))
    return fail(JXF_ERR_INVALID, "invalid arguments");
  if (n == 0) return JXF_OK;
  for (int i = 0; i < n; ++i)
    if (face[i] < 0 || face[i] > 5) return fail(JXF_ERR_INVALID, "face[%d] = %d", i, face[i]);
  DeviceGuard dg(m->device);
  std::vector<int2> per[6];
  for (int i = 0; i < n; ++i) per[face[i]].push_back(make_int2(i, 0));
  std::vector<int2> cells;
  std::vector<int> tf;
  band_tiles(per, cells, tf);
  float* d_rows = nullptr;
  float* d_out = nullptr;
  int2* d_cells = nullptr;
  int* d_tf = nullptr;
  int64_t tally = 0;
  int rc = dmalloc(&d_rows, (size_t)n * band::kIn, &tally);
  if (rc == JXF_OK) rc = dmalloc(&d_out, cells.size() * band::kOut, &tally);
  if (rc == JXF_OK) rc = upload(&d_cells, cells, &tally);
  if (rc == JXF_OK) rc = upload(&d_tf, tf, &tally);
  if (rc == JXF_OK &&
      cudaMemcpy(d_rows, feat, (size_t)n * band::kIn * 4, cudaMemcpyHostToDevice) != cudaSuccess)
    rc = fail(JXF_ERR_CUDA, "copy of feature rows failed");
  if (rc == JXF_OK) {
    band::InferArgs a{};
    a.cells = d_cells;
    a.tile_face = d_tf;
    a.n_tiles = (int)tf.size();
    a.wimg = m->d_wimg;
    a.params = m->d_params;
    a.delta = d_out;
    a.rows = d_rows;
    a.err = m->d_err;
    a.wait_ns = wait_limit_ns();
    band::k_band_infer<band::SRC_ROWS><<<band_ctas(a.n_tiles, m->device), 128, band::kInfSmem>>>(a);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) rc = fail(JXF_ERR_CUDA, "band eval: %s", cudaGetErrorString(e));
  }
  if (rc == JXF_OK) {
    std::vector<float> h(cells.size() * band::kOut);
    if (cudaMemcpy(h.data(), d_out, h.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = fail(JXF_ERR_CUDA, "copy of outputs failed");
    for (size_t i = 0; rc == JXF_OK && i < cells.size(); ++i)
      if (cells[i].x >= 0)
        for (int o = 0; o < band::kOut; ++o) out[(size_t)cells[i].x * band::kOut + o] = h[i * 6 + o];
  }
  dfree(d_rows);
  dfree(d_out);
  dfree(d_cells);
  dfree(d_tf);
  if (rc == JXF_OK) rc = jxf_band_check_error(m, nullptr);
  return rc;
}

int jxf_band_collect(jxf_band* m, float* const* fields, int32_t nx, int32_t ny, int32_t nz,
                     const float* const* ref, int32_t rnx, int32_t rny, int32_t rnz, int32_t ox,
                     int32_t oy, int32_t oz, void* stream) {
  if (!m || !fields || !ref) return fail(JXF_ERR_INVALID, "null argument");
  TRY(band_check_dims(nx, ny, nz));
  if (ox < 0 || oy < 0 || oz < 0 || ox + nx > rnx || oy + ny > rny || oz + nz > rnz)
    return fail(JXF_ERR_INVALID, "the %d x %d x %d box at (%d, %d, %d) is outside the %d x %d x %d "
                "reference grid", nx, ny, nz, ox, oy, oz, rnx, rny, rnz);
  for (int c = 0; c < 6; ++c)
    if (!fields[c] || !ref[c]) return fail(JXF_ERR_INVALID, "null field pointer %d", c);
  DeviceGuard dg(m->device);
  cudaStream_t st = (cudaStream_t)stream;
  // earlier collects on `st` may still write the row buffers or read d_cells
  CUDA_TRY(cudaStreamSynchronize(st));
  std::vector<int> per[6];
  band_cells(nx, ny, nz, per);
  std::vector<int> all;
  band::CollectArgs a{};
  a.first[0] = 0;
  for (int f = 0; f < 6; ++f) {
    all.insert(all.end(), per[f].begin(), per[f].end());
    a.first[f + 1] = (int)all.size();
    TRY(band_grow(m, f, m->rows[f] + (long long)per[f].size()));
    a.base[f] = m->rows[f];
    a.feat[f] = m->feat[f];
    a.tgt[f] = m->tgt[f];
    a.w[f] = m->w[f];
  }
  if (all.size() > m->cells_cap) {
    dfree(m->d_cells);
    TRY(dmalloc(&m->d_cells, all.size(), &m->bytes));
    m->cells_cap = all.size();
  }
  CUDA_TRY(cudaMemcpy(m->d_cells, all.data(), all.size() * 4, cudaMemcpyHostToDevice));
  for (int c = 0; c < 6; ++c) {
    a.t.f[c] = fields[c];
    a.ref[c] = ref[c];
  }
  a.t.nx = nx;
  a.t.ny = ny;
  a.t.nz = nz;
  a.rnx = rnx;
  a.rny = rny;
  a.rnz = rnz;
  a.ox = ox;
  a.oy = oy;
  a.oz = oz;
  a.cells = m->d_cells;
  band::k_band_collect<<<((int)all.size() + 127) / 128, 128, 0, st>>>(a);
  CUDA_TRY(cudaGetLastError());
  for (int f = 0; f < 6; ++f) m->rows[f] += (long long)per[f].size();
  return JXF_OK;
}

int jxf_band_dataset_size(jxf_band* m, int64_t* rows) {
  if (!m || !rows) return fail(JXF_ERR_INVALID, "null argument");
  for (int f = 0; f < 6; ++f) rows[f] = m->rows[f];
  return JXF_OK;
}

int jxf_band_dataset_clear(jxf_band* m) {
  if (!m) return fail(JXF_ERR_INVALID, "null handle");
  for (int f = 0; f < 6; ++f) m->rows[f] = 0;
  return JXF_OK;
}

int jxf_band_dataset_get(jxf_band* m, int32_t face, int64_t first, int64_t count, uint16_t* feat,
                         float* target, float* weight) {
  if (!m || face < 0 || face > 5) return fail(JXF_ERR_INVALID, "invalid handle or face");
  if (first < 0 || count < 0 || first + count > m->rows[face])
    return fail(JXF_ERR_INVALID, "rows [%lld, %lld) outside the %lld rows of face %d",
                (long long)first, (long long)(first + count), m->rows[face], face);
  if (count == 0) return JXF_OK;
  DeviceGuard dg(m->device);
  CUDA_TRY(cudaDeviceSynchronize());
  if (feat)
    CUDA_TRY(cudaMemcpy(feat, m->feat[face] + first * band::kInP, count * band::kInP * 2,
                        cudaMemcpyDeviceToHost));
  if (target)
    CUDA_TRY(cudaMemcpy(target, m->tgt[face] + first * band::kOut, count * band::kOut * 4,
                        cudaMemcpyDeviceToHost));
  if (weight)
    CUDA_TRY(cudaMemcpy(weight, m->w[face] + first, count * 4, cudaMemcpyDeviceToHost));
  return JXF_OK;
}

int jxf_band_grad(jxf_band* m, float* grad, float* loss, void* stream) {
  if (!m) return fail(JXF_ERR_INVALID, "null handle");
  DeviceGuard dg(m->device);
  cudaStream_t st = (cudaStream_t)stream;
  double ws[6];
  TRY(band_weight_sums(m, ws, st));
  if (m->loss_cap < 1) {
    dfree(m->d_loss);
    TRY(dmalloc(&m->d_loss, 6, &m->bytes));
    m->loss_cap = 1;
  }
  band::TrainArgs a = band_train_args(m);
  a.random = 0;
  for (int f = 0; f < 6; ++f) {
    a.tiles[f] = (int)((m->rows[f] + band::kTile - 1) / band::kTile);
    a.scale[f] = ws[f] > 0.0 ? (float)(1.0 / ws[f]) : 0.0f;
  }
  a.loss = m->d_loss;
  CUDA_TRY(cudaMemsetAsync(m->d_grad, 0, 6 * (size_t)band::kParams * 4, st));
  CUDA_TRY(cudaMemsetAsync(m->d_loss, 0, 6 * 4, st));
  TRY(band_train_pass(m, a, st));
  if (grad)
    CUDA_TRY(cudaMemcpyAsync(grad, m->d_grad, 6 * (size_t)band::kParams * 4,
                             cudaMemcpyDeviceToHost, st));
  if (loss) CUDA_TRY(cudaMemcpyAsync(loss, m->d_loss, 6 * 4, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return jxf_band_check_error(m, stream);
}

int jxf_band_train(jxf_band* m, int32_t iters, int32_t batch_rows, float lr, uint64_t seed,
                   float* loss, void* stream) {
  if (!m) return fail(JXF_ERR_INVALID, "null handle");
  if (iters < 0 || batch_rows < 1) return fail(JXF_ERR_INVALID, "iters >= 0, batch_rows >= 1");
  if (iters == 0) return JXF_OK;
  DeviceGuard dg(m->device);
  cudaStream_t st = (cudaStream_t)stream;
  double ws[6];
  TRY(band_weight_sums(m, ws, st));
  if (m->loss_cap < (size_t)iters) {
    dfree(m->d_loss);
    TRY(dmalloc(&m->d_loss, (size_t)iters * 6, &m->bytes));
    m->loss_cap = (size_t)iters;
  }
  CUDA_TRY(cudaMemsetAsync(m->d_loss, 0, (size_t)iters * 6 * 4, st));
  const int tiles = (batch_rows + band::kTile - 1) / band::kTile;
  band::TrainArgs a = band_train_args(m);
  a.random = 1;
  for (int f = 0; f < 6; ++f) {
    a.tiles[f] = m->rows[f] > 0 ? tiles : 0;
    const double mean = m->rows[f] > 0 ? ws[f] / (double)m->rows[f] : 0.0;
    a.scale[f] = mean > 0.0 ? (float)(1.0 / ((double)tiles * band::kTile * mean)) : 0.0f;
  }
  const float b1 = 0.9f, b2 = 0.999f;
  for (int it = 0; it < iters; ++it) {
    a.seed = band::mix64(seed + 0x9e3779b97f4a7c15ull * (unsigned long long)(it + 1));
    a.loss = m->d_loss + (size_t)it * 6;
    CUDA_TRY(cudaMemsetAsync(m->d_grad, 0, 6 * (size_t)band::kParams * 4, st));
    TRY(band_train_pass(m, a, st));
    m->adam_t += 1;
    const float c1 = (float)(1.0 - std::pow(0.9, (double)m->adam_t));
    const float c2 = (float)(1.0 - std::pow(0.999, (double)m->adam_t));
    band::k_band_adam<<<(6 * band::kParams + 255) / 256, 256, 0, st>>>(
        m->d_params, m->d_grad, m->d_m1, m->d_m2, 6 * band::kParams, lr, b1, b2, 1e-8f, c1, c2);
    TRY(band_pack(m, st));
  }
  CUDA_TRY(cudaGetLastError());
  if (loss) {
    std::vector<float> h((size_t)iters * 6);
    CUDA_TRY(cudaMemcpyAsync(h.data(), m->d_loss, h.size() * 4, cudaMemcpyDeviceToHost, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    for (int it = 0; it < iters; ++it) {
      float s = 0.0f;
      for (int f = 0; f < 6; ++f) s += h[(size_t)it * 6 + f];
      loss[it] = s;
    }
  }
  return jxf_band_check_error(m, stream);
}

int jxf_band_check_error(jxf_band* m, void* stream) {
  if (!m) return fail(JXF_ERR_INVALID, "null handle");
  DeviceGuard dg(m->device);
  cudaStream_t st = (cudaStream_t)stream;
  int h[4] = {0, 0, 0, 0};
  CUDA_TRY(cudaMemcpyAsync(h, m->d_err, 16, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  CUDA_TRY(cudaGetLastError());
  if (h[0] != 0) {
    CUDA_TRY(cudaMemsetAsync(m->d_err, 0, 16, st));
    CUDA_TRY(cudaStreamSynchronize(st));
    return fail(JXF_ERR_TIMEOUT,
                "a tensor-core step did not complete within the wait limit (code 0x%x, block %d, "
                "face %d, thread %d)",
                h[0], h[1], h[2], h[3]);
  }
  return JXF_OK;
}

int jxf_batch3d_set_band(jxf_batch3d* b, jxf_band* m) {
  if (!b) return fail(JXF_ERR_INVALID, "null batch");
  DeviceGuard dg(b->device);
  if (b->graph) {
    cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
  }
  band_release(b->band);
  if (!m) return JXF_OK;
  return band_attach(b->grids, m, b->device, &b->bytes, b->band);
}

int jxf_grid3d_set_band(jxf_grid3d* g, jxf_band* m) {
  if (!g) return fail(JXF_ERR_INVALID, "null grid");
  DeviceGuard dg(g->d.device);
  CUDA_TRY(cudaDeviceSynchronize());
  band_release(g->band);
  if (!m) return JXF_OK;
  if (g->slab) return fail(JXF_ERR_INVALID, "a learned band runs on a whole grid");
  std::vector<jxf_grid3d*> one{g};
  return band_attach(one, m, g->d.device, &g->bytes, g->band);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Adjoint (permittivity gradients of probe objectives)
// ---------------------------------------------------------------------------

namespace {

size_t psi_size(const jxf_grid3d* g, int id) {
  static const int axis_of[PSI_COUNT] = {1, 2, 2, 0, 0, 1, 1, 2, 2, 0, 0, 1};
  const int ax = axis_of[id];
  if (g->mode != MODE_CPML) return 0;
  if (ax == 0) return (size_t)g->L[0] * g->d.ny * g->d.nz;
  if (ax == 1) return (size_t)g->d.nx * g->L[1] * g->d.nz;
  return (size_t)g->d.nx * g->d.ny * g->L[2];
}

template <class T>
int ensure_buf(T** p, size_t* cap, size_t count, int64_t* tally) {
  if (*cap >= count && *p) return JXF_OK;
  dfree(*p);
  *cap = 0;
  TRY(dmalloc(p, count, tally));
  *cap = count;
  return JXF_OK;
}

// Several device-to-device copies of float arrays in one launch (the
// recompute of an adjoint segment keeps H and the E psi after every step:
// one launch instead of one copy per array).
struct CopyList {
  const float* src[18];
  float* dst[18];
  long long end[18];  // cumulative element counts
  int n;
};
__global__ void k_copy_many(const __grid_constant__ CopyList c) {
  const long long total = c.end[c.n - 1];
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    int k = 0;
    while (i >= c.end[k]) ++k;
    const long long j = i - (k ? c.end[k - 1] : 0);
    c.dst[k][j] = c.src[k][j];
  }
}
struct CopyBatch {
  CopyList c{};
  bool overflow = false;
  void add(float* dst, const float* src, size_t n) {
    if (n == 0) return;
    if (c.n == (int)(sizeof(c.src) / sizeof(c.src[0]))) {
      overflow = true;
      return;
    }
    c.src[c.n] = src;
    c.dst[c.n] = dst;
    c.end[c.n] = (c.n ? c.end[c.n - 1] : 0) + (long long)n;
    ++c.n;
  }
  int launch(cudaStream_t st) {
    if (overflow) return fail(JXF_ERR_INVALID, "internal: more than 18 arrays in one copy batch");
    if (c.n == 0) return JXF_OK;
    const long long total = c.end[c.n - 1];
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148LL * 8);
    k_copy_many<<<blocks, 256, 0, st>>>(c);
    CUDA_TRY(cudaGetLastError());
    return JXF_OK;
  }
};

// copy the current state (fields + psi) to / from one checkpoint slot
int ckpt_copy(jxf_grid3d* g, float* slot, bool save, cudaStream_t st) {
  const size_t n = (size_t)g->n;
  size_t off = 0;
  CopyBatch cb;
  for (int k = 0; k < 6; ++k) {
    float* f = g->f[g->cur][k];
    cb.add(save ? slot + off : f, save ? f : slot + off, n);
    off += n;
  }
  for (int k = 0; k < PSI_COUNT; ++k) {
    const size_t sz = psi_size(g, k);
    float* q = g->psi[g->cur][k];
    cb.add(save ? slot + off : q, save ? q : slot + off, sz);
    off += sz;
  }
  return cb.launch(st);
}

}  // namespace

extern "C" int jxf_grid3d_adjoint_forward(jxf_grid3d* g, int32_t n_steps,
                                          int32_t checkpoint_every, float* probe_out,
                                          void* stream) {
  if (!g) return fail(JXF_ERR_INVALID, "null handle");
  if (n_steps < 1) return fail(JXF_ERR_INVALID, "n_steps must be >= 1");
  if (g->slab) return fail(JXF_ERR_INVALID, "the adjoint runs on whole grids, not x-slabs");
  if (g->mode == MODE_PERIODIC)
    return fail(JXF_ERR_INVALID, "the adjoint supports ABSORBING, PEC and CPML boundaries");
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  const int K = checkpoint_every > 0 ? checkpoint_every
                                     : std::max(1, (int)std::ceil(std::sqrt((double)n_steps)));
  const int nseg = (n_steps + K - 1) / K;
  size_t state = 6 * (size_t)g->n, segstate = 3 * (size_t)g->n;
  for (int k = 0; k < PSI_COUNT; ++k) state += psi_size(g, k);
  for (int k = PSI_EXY; k < PSI_COUNT; ++k) segstate += psi_size(g, k);
  TRY(ensure_buf(&g->adj_ck, &g->adj_ck_cap, state * nseg, &g->bytes));
  TRY(jxf_grid3d_reset(g, stream));
  const int np = g->n_probes;
  for (int s = 0; s < nseg; ++s) {
    const int start = s * K, len = std::min(K, n_steps - start);
    TRY(ckpt_copy(g, g->adj_ck + (size_t)s * state, true, st));
    TRY(jxf_grid3d_step(g, len, probe_out ? probe_out + (size_t)start * np : nullptr, stream));
  }
  g->adj_n = n_steps;
  g->adj_k = K;
  g->adj_nseg = nseg;
  g->adj_state = state;
  g->adj_segstate = segstate;
  return JXF_OK;
}

extern "C" int jxf_grid3d_adjoint_backward(jxf_grid3d* g, const float* probe_grad,
                                           float* grad_eps, void* stream) {
  if (!g || !grad_eps) return fail(JXF_ERR_INVALID, "null argument");
  if (g->adj_n < 1) return fail(JXF_ERR_INVALID, "call jxf_grid3d_adjoint_forward first");
  if (g->n_probes > 0 && !probe_grad) return fail(JXF_ERR_INVALID, "probe_grad is null");
  DeviceGuard dg(g->d.device);
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = (size_t)g->n;
  const int K = g->adj_k, N = g->adj_n;
  size_t psi_tot = 0;
  for (int k = 0; k < PSI_COUNT; ++k) psi_tot += psi_size(g, k);
  TRY(ensure_buf(&g->adj_sg, &g->adj_sg_cap, g->adj_segstate * K, &g->bytes));
  TRY(ensure_buf(&g->adj_l, &g->adj_l_cap, 18 * n + psi_tot, &g->bytes));
  TRY(ensure_buf(&g->adj_g, &g->adj_g_cap, n, &g->bytes));
  CUDA_TRY(cudaMemsetAsync(g->adj_l, 0, (18 * n + psi_tot) * 4, st));
  CUDA_TRY(cudaMemsetAsync(g->adj_g, 0, n * 8, st));

  Adj3D a{};
  a.nx = g->d.nx;
  a.ny = g->d.ny;
  a.nz = g->d.nz;
  a.div_nz = make_fastdiv((uint32_t)g->d.nz);
  a.div_ny = make_fastdiv((uint32_t)g->d.ny);
  a.idx32 = ((long long)g->d.nx * g->d.ny * g->d.nz) < (1ll << 32) ? 1 : 0;
  a.a = (float)g->coef_h;
  a.cb_const = (float)g->coef_e;
  a.cb = g->cb;
  for (int ax = 0; ax < 3; ++ax) {
    a.damp[ax] = g->damp[ax];
    for (int t = 0; t < TAB_COUNT; ++t) a.pml.tab[ax][t] = g->tab[ax][t];
    a.pml.L[ax] = g->L[ax];
    a.pml.P[ax] = g->P[ax];
  }
  float* lp = g->adj_l;
  Lam6 lam;
  for (int c = 0; c < 3; ++c) {
    a.lE[c] = lp + c * n;
    a.lH[c] = lp + (3 + c) * n;
    lam.f[c] = a.lE[c];
    lam.f[3 + c] = a.lH[c];
  }
  {
    size_t off = 6 * n;
    for (int k = 0; k < PSI_COUNT; ++k) {
      a.lpsi[k] = psi_size(g, k) ? lp + off : nullptr;
      off += psi_size(g, k);
    }
    for (int k = 0; k < 6; ++k) {
      a.db[k] = lp + off + k * n;
      a.dh[k] = lp + off + (6 + k) * n;
    }
  }
  a.gcb = g->adj_g;
  const int threads = 256;
  const int blocks = (int)std::min<long long>(((long long)n + threads - 1) / threads, 148LL * 16);
  const int np = g->n_probes;

  for (int s = g->adj_nseg - 1; s >= 0; --s) {
    const int start = s * K, len = std::min(K, N - start);
    // recompute the segment, keeping (H, psiE) after every step
    TRY(ckpt_copy(g, g->adj_ck + (size_t)s * g->adj_state, false, st));
    g->step = start;
    for (int k = 0; k < len; ++k) {
      TRY(jxf_grid3d_step(g, 1, nullptr, stream));
      float* slot = g->adj_sg + (size_t)k * g->adj_segstate;
      size_t off = 0;
      CopyBatch cb;
      for (int c = 0; c < 3; ++c) {
        cb.add(slot + off, g->f[g->cur][3 + c], n);
        off += n;
      }
      for (int q = PSI_EXY; q < PSI_COUNT; ++q) {
        const size_t sz = psi_size(g, q);
        cb.add(slot + off, g->psi[g->cur][q], sz);
        off += sz;
      }
      TRY(cb.launch(st));
    }
    // adjoint steps, last to first
    for (int k = len - 1; k >= 0; --k) {
      const int step_n = start + k;
      if (np > 0) {
        k3a_seed<<<1, 32, 0, st>>>(lam, g->d_probe_cell, g->d_probe_comp, np,
                                   probe_grad + (size_t)step_n * np);
      }
      const float* slot = g->adj_sg + (size_t)k * g->adj_segstate;
      size_t off = 0;
      for (int c = 0; c < 3; ++c) {
        a.fh[c] = slot + off;
        off += n;
      }
      for (int q = PSI_EXY; q < PSI_COUNT; ++q) {
        const size_t sz = psi_size(g, q);
        a.fpsiE[q - PSI_EXY] = sz ? slot + off : nullptr;
        off += sz;
      }
      if (g->mode == MODE_CPML) {
        k3a_e<MODE_CPML><<<blocks, threads, 0, st>>>(a);
        k3a_h<MODE_CPML><<<blocks, threads, 0, st>>>(a);
      } else {
        k3a_e<MODE_ABSORB><<<blocks, threads, 0, st>>>(a);
        k3a_h<MODE_ABSORB><<<blocks, threads, 0, st>>>(a);
      }
      k3a_e2<<<blocks, threads, 0, st>>>(a);
      CUDA_TRY(cudaGetLastError());
    }
  }
  k3a_finish<<<blocks, threads, 0, st>>>(g->adj_g, g->cb, (float)g->coef_e, g->coef_e, grad_eps,
                                         (long long)n);
  CUDA_TRY(cudaGetLastError());
  // leave the grid at its initial state
  TRY(ckpt_copy(g, g->adj_ck, false, st));
  g->step = 0;
  return JXF_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free entry point
// ---------------------------------------------------------------------------
//
// For callers that cannot call cudaMalloc: code that runs inside a memory
// pool owned by another framework (for example an XLA custom call, which must
// not grab device memory behind the pool's back), or hosts that forbid
// allocation once they are running.  The TMA step
// kernel needs a second set of six field buffers to ping-pong into, plus the
// damping tables and an error word; here they live in one fixed device array
// that every GPU loading this library holds until the process exits.

namespace {

constexpr long long kNoAllocMaxCells = 262144;  // 64^3
constexpr int kNoAllocMaxAxis = 4096;
constexpr size_t kNoAllocFieldBytes = 6 * (size_t)kNoAllocMaxCells * sizeof(float);
constexpr size_t kNoAllocTableBytes = 3 * (size_t)kNoAllocMaxAxis * sizeof(float);
constexpr size_t kNoAllocBytes = kNoAllocFieldBytes + kNoAllocTableBytes + 256;

// Device scratch of jxf_grid3d_run_noalloc: [6 fields][max cells] float32,
// then [3 axes][max axis] damping factors, then 4 error words.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[128] = {};

// Device address of the scratch array on `dev` (the current device).  The
// host-side symbol is only a stand-in for the device array, so its address
// is resolved once per device here and passed to the kernel.
int noalloc_scratch(int dev, unsigned char** out) {
  if (dev < 0 || dev >= 128) return fail(JXF_ERR_INVALID, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess || ptr == nullptr)
      return fail(JXF_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s", cudaGetErrorString(e));
    g_noalloc_addr[dev] = ptr;
  }
  *out = static_cast<unsigned char*>(g_noalloc_addr[dev]);
  return JXF_OK;
}

}  // namespace

extern "C" int jxf_grid3d_run_noalloc(const jxf_noalloc_desc* desc, float* const* fields,
                                      const float* cb, int32_t n_steps, void* stream) {
  if (!desc || !fields) return fail(JXF_ERR_INVALID, "null argument");
  const jxf_noalloc_desc d = *desc;
  for (int k = 0; k < 6; ++k)
    if (!fields[k]) return fail(JXF_ERR_INVALID, "field pointer %d is null", k);
  // the TMA tensor maps need 16-byte aligned base addresses
  for (int k = 0; k < 6; ++k)
    if (reinterpret_cast<uintptr_t>(fields[k]) % 16 != 0)
      return fail(JXF_ERR_INVALID, "field pointer %d is not 16-byte aligned", k);
  if (cb && reinterpret_cast<uintptr_t>(cb) % 16 != 0)
    return fail(JXF_ERR_INVALID, "cb pointer is not 16-byte aligned");
  if (n_steps < 0) return fail(JXF_ERR_INVALID, "n_steps must be >= 0");
  if (d.nx < 2 || d.ny < 2 || d.nz < 2)
    return fail(JXF_ERR_INVALID, "grid must be at least 2 cells per axis");
  if (d.nz % 4 != 0) return fail(JXF_ERR_INVALID, "nz must be a multiple of 4 (got %d)", d.nz);
  if (d.nx > kNoAllocMaxAxis || d.ny > kNoAllocMaxAxis || d.nz > kNoAllocMaxAxis ||
      (long long)d.nx * d.ny * d.nz > kNoAllocMaxCells)
    return fail(JXF_ERR_INVALID,
                "grid %dx%dx%d exceeds the allocation-free limit (%lld cells, %d per axis)", d.nx,
                d.ny, d.nz, kNoAllocMaxCells, kNoAllocMaxAxis);
  if (d.boundary != JXF_BND_ABSORBING && d.boundary != JXF_BND_PEC)
    return fail(JXF_ERR_INVALID, "allocation-free steps support ABSORBING and PEC boundaries");
  if (!(d.dx > 0)) return fail(JXF_ERR_INVALID, "dx must be positive");
  if (d.pml_layers < 0) return fail(JXF_ERR_INVALID, "pml_layers must be >= 0");
  if (n_steps == 0) return JXF_OK;
  DeviceGuard dg(d.device);
  if (!dg.ok) return fail(JXF_ERR_CUDA, "cannot select device %d", d.device);
  unsigned char* base = nullptr;
  TRY(noalloc_scratch(d.device, &base));
  cudaStream_t st = (cudaStream_t)stream;
  float* fB = reinterpret_cast<float*>(base);
  float* tabs = reinterpret_cast<float*>(base + kNoAllocFieldBytes);
  int* err = reinterpret_cast<int*>(base + kNoAllocFieldBytes + kNoAllocTableBytes);
  const long long n = (long long)d.nx * d.ny * d.nz;
  const double dt = d.dt > 0 ? d.dt : 0.99 * d.dx / (kC0 * std::sqrt(3.0));

  // damping factors (ones for PEC) into the scratch tables; the error word
  // keeps the previous call's value, so clear it
  const int dims[3] = {d.nx, d.ny, d.nz};
  for (int ax = 0; ax < 3; ++ax) {
    std::vector<float> t = d.boundary == JXF_BND_ABSORBING
                               ? damping_table(dims[ax], d.pml_layers, d.dx, dt, 3)
                               : std::vector<float>(dims[ax], 1.0f);
    CUDA_TRY(cudaMemcpyAsync(tabs + (size_t)ax * kNoAllocMaxAxis, t.data(), t.size() * 4,
                             cudaMemcpyHostToDevice, st));
  }
  CUDA_TRY(cudaMemsetAsync(err, 0, 16, st));

  const int cfg = 0;
  const TmaConfig& c = tma_configs()[cfg];
  const int chunk = n >= (1LL << 17) ? 16 : 8;
  float* set[2][6];
  for (int k = 0; k < 6; ++k) {
    set[0][k] = fields[k];
    set[1][k] = fB + (size_t)k * n;
  }
  Maps3D maps[2];
  for (int s = 0; s < 2; ++s) {
    for (int k = 0; k < 3; ++k) {
      TRY(encode_map(&maps[s].e[k], set[s][k], d.nx, d.ny, d.nz, c.tz + 8, c.ty + 2));
      TRY(encode_map(&maps[s].h[k], set[s][3 + k], d.nx, d.ny, d.nz, c.tz + 4, c.ty + 1));
    }
    if (cb) {
      TRY(encode_map(&maps[s].cb, cb, d.nx, d.ny, d.nz, c.tz, c.ty));
    } else {
      maps[s].cb = maps[s].e[0];
    }
  }
  Step3D p{};
  p.drop_stage = -1;
  p.nx = d.nx;
  p.ny = d.ny;
  p.nz = d.nz;
  p.gnx = d.nx;  // a whole grid: gx0 = x_lo = 0
  p.x_hi = d.nx;
  p.a = (float)(dt / (kMu0 * d.dx));
  p.cb_const = (float)(dt / (kEps0 * d.dx));
  p.cb = cb;
  for (int ax = 0; ax < 3; ++ax) p.damp[ax] = tabs + (size_t)ax * kNoAllocMaxAxis;
  for (int ax = 0; ax < 3; ++ax) {
    for (int t = 0; t < TAB_COUNT; ++t) p.pml.tab[ax][t] = p.damp[ax];
    p.pml.L[ax] = 0;
    p.pml.P[ax] = -1;
  }
  p.err = err;
  p.wait_ns = wait_limit_ns();
  p.x_chunk = chunk;
  p.ntiles_z = (d.nz + c.tz - 1) / c.tz;
  p.ntiles_y = (d.ny + c.ty - 1) / c.ty;
  TmaKernel k = c.k[0][cb ? 1 : 0];
  {
    static std::mutex mu;
    std::lock_guard<std::mutex> lk(mu);
    CUDA_TRY(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)c.smem[0]));
  }
  const dim3 grid(p.ntiles_z, p.ntiles_y, (d.nx + chunk - 1) / chunk);
  int cur = 0;
  for (int s = 0; s < n_steps; ++s) {
    for (int q = 0; q < 6; ++q) {
      p.in[q] = set[cur][q];
      p.out[q] = set[cur ^ 1][q];
    }
    p.step = s;
    k<<<grid, c.threads, c.smem[0], st>>>(p, maps[cur]);
    CUDA_TRY(cudaGetLastError());
    cur ^= 1;
  }
  if (cur == 1)  // odd step count: the result sits in the scratch set
    for (int q = 0; q < 6; ++q)
      CUDA_TRY(cudaMemcpyAsync(fields[q], set[1][q], (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
  int h[4] = {0, 0, 0, 0};
  CUDA_TRY(cudaMemcpyAsync(h, err, 16, cudaMemcpyDeviceToHost, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  if (h[0] != 0)
    return fail(JXF_ERR_TIMEOUT, "a staged copy did not arrive within the wait limit (block %d)",
                h[1]);
  return JXF_OK;
}
