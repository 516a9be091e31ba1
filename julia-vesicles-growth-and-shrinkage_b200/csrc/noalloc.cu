// Allocation-free inverse 2D real FFT (FP32) for callers that cannot call
// cudaMalloc: code that runs inside a larger application whose GPU memory is
// owned by someone else (a memory pool, a captured or replayed stream, an
// embedding runtime that forbids device allocations) or that must never block
// on the allocator.  The caller passes its own device input and output; the
// one intermediate buffer this transform needs (the spectrum after the
// y/column pass) and the twiddle table live in file-scope __device__ arrays
// of a fixed size, reserved once per GPU when the library is loaded and held
// until the process exits.
//
// Same arithmetic as the handle path's irfft (column pass, then row c2r pass
// that keeps only Re of the kx=0 and kx=Nx/2 bins), with one fixed kernel
// variant instead of the autotuned one.
#include "../../include/vsav.h"
#include "fft.cuh"

#include <mutex>
#include <string>
#include <vector>

namespace vsav {

// scratch: the column-pass output, nf * Ny * (Nx/2+1) complex floats at most
constexpr long long NOALLOC_MAX_COMPLEX = 1LL << 20;        // 1 Mi complex = 8 MiB
constexpr int NOALLOC_MAX_N = 2048;                         // largest Nx or Ny
static __device__ __align__(256) float2 g_noalloc_scratch[NOALLOC_MAX_COMPLEX];
// twiddles tab[n + m] = exp(-2 pi i m / n) for n = 1 .. NOALLOC_MAX_N
static __device__ __align__(256) float2 g_noalloc_tab[2 * NOALLOC_MAX_N];

namespace {

// Per-device set-up record.  The table has a fixed size and never moves, and
// callers copy the two addresses out while they hold the lock, so a first
// call on another device (from another host thread) cannot invalidate them.
constexpr int NOALLOC_MAX_DEVICES = 64;
struct DevSetup {
  bool done = false;
  float2* scratch = nullptr;   // device addresses of the two arrays on this device
  float2* tab = nullptr;
};
std::mutex g_setup_mutex;
DevSetup g_setup[NOALLOC_MAX_DEVICES];
thread_local std::string g_noalloc_error;

int fail(const std::string& m, int code) { g_noalloc_error = m; return code; }

// once per device, with that device current: resolve the device addresses of
// the file-scope arrays (a host-side use of the array names would be a host
// stand-in, not a device address) and fill the twiddle table.  The addresses
// are returned by value.
int setup_device(int dev, float2*& scratch, float2*& tab) {
  if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
    return fail("device ordinal " + std::to_string(dev) + " is beyond the " + std::to_string(NOALLOC_MAX_DEVICES) +
                    " devices this entry point supports",
                VSAV_E_INVALID);
  std::lock_guard<std::mutex> lk(g_setup_mutex);
  DevSetup& d = g_setup[dev];
  if (!d.done) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail(std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e), VSAV_E_CUDA);
    float2* sp = (float2*)p;
    e = cudaGetSymbolAddress(&p, g_noalloc_tab);
    if (e != cudaSuccess) return fail(std::string("cudaGetSymbolAddress(twiddles): ") + cudaGetErrorString(e), VSAV_E_CUDA);
    float2* tp = (float2*)p;
    std::vector<float2> ht(2 * NOALLOC_MAX_N);
    for (int n = 1; n <= NOALLOC_MAX_N; n <<= 1)
      for (int m = 0; m < n; ++m) {
        long double a = -2.0L * 3.14159265358979323846264338327950288L * (long double)m / (long double)n;
        long double cr = cosl(a), ci = sinl(a);
        if (4 * m % n == 0) { int q = 4 * m / n; cr = (q == 0) ? 1 : (q == 2 ? -1 : 0); ci = (q == 1) ? -1 : (q == 3 ? 1 : 0); }
        ht[n + m] = make_float2((float)cr, (float)ci);
      }
    e = cudaMemcpyToSymbol(g_noalloc_tab, ht.data(), ht.size() * sizeof(float2));
    if (e != cudaSuccess) return fail(std::string("twiddle upload: ") + cudaGetErrorString(e), VSAV_E_CUDA);
    d.scratch = sp;
    d.tab = tp;
    d.done = true;
  }
  scratch = d.scratch;
  tab = d.tab;
  return VSAV_OK;
}

int ilog2i(int n) { int l = 0; while ((1 << l) < n) ++l; return l; }
bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

}  // namespace
}  // namespace vsav

using namespace vsav;

// The two launches go through cudaLaunchKernel, whose return value is the
// status of that launch alone: an error that the caller's earlier CUDA work
// left pending on this thread is neither reported as ours nor cleared.
extern "C" int vsav_irfft2d_f32_noalloc(const float* spec, float* out, int32_t nf, int32_t Nx, int32_t Ny, double Lx,
                                        double Ly, int32_t mult, void* stream) {
  constexpr int E = 8, NT = 256;
  g_noalloc_error.clear();
  if (!spec || !out) return fail("null input or output pointer", VSAV_E_INVALID);
  if (!pow2(Nx) || Nx < 32 || Nx > NOALLOC_MAX_N || !pow2(Ny) || Ny < E || Ny > NOALLOC_MAX_N)
    return fail("Nx must be a power of two in [32, 2048] and Ny a power of two in [8, 2048]", VSAV_E_INVALID);
  if (!(mult == M_ONE || mult == M_DX || mult == M_DY || mult == M_LAP || mult == M_BIH))
    return fail("mult must be 0 (none), 1 (d/dx), 2 (d/dy), 4 (Laplacian) or 5 (biharmonic)", VSAV_E_INVALID);
  if (!(Lx > 0) || !(Ly > 0)) return fail("Lx and Ly must be > 0", VSAV_E_INVALID);
  const int nkx = Nx / 2 + 1;
  const long long need = (long long)nf * Ny * nkx;
  if (nf < 1 || need > NOALLOC_MAX_COMPLEX)
    return fail("nf * Ny * (Nx/2+1) = " + std::to_string(need) + " complex values exceeds the fixed scratch of " +
                    std::to_string(NOALLOC_MAX_COMPLEX) + " (8 MiB); split the batch",
                VSAV_E_INVALID);
  if (((uintptr_t)spec | (uintptr_t)out) & 7) return fail("input and output must be 8-byte aligned", VSAV_E_INVALID);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(std::string("cudaGetDevice: ") + cudaGetErrorString(e), VSAV_E_CUDA);
  float2* scratch = nullptr;
  float2* tab = nullptr;
  int rc = setup_device(dev, scratch, tab);
  if (rc != VSAV_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // column (y) pass: spec -> scratch, both in the caller's unpadded layout [nf][Ny][nkx]
  ColArgs a{};
  a.geo = 0; a.Nx = Nx; a.Ny = Ny; a.Nz = 1; a.kp = nkx;
  a.kxs = 2 * M_PI / Lx; a.kys = 2 * M_PI / Ly; a.kzs = 0.0;
  a.fkxs = (float)a.kxs; a.fkys = (float)a.kys; a.fkzs = 0.f;
  a.logL = ilog2i(Ny); a.S = nkx; a.W = nkx; a.O = (long long)Ny * nkx; a.kpv = nkx; a.nkv = nkx;
  int TW = std::max(1, E * NT / Ny);
  while (TW > 1 && TW / 2 >= a.W) TW /= 2;
  a.TW = TW; a.logTW = ilog2i(TW); a.tiles = (a.W + TW - 1) / TW;
  const int thr_c = std::max(TW, TW * Ny / E);
  const size_t sm_c = 2 * (size_t)col_tile_elems(Ny, TW, ilog2i(E)) * sizeof(float2);
  const void* kc = (const void*)k_cols<float, E, NT, true>;
  if (sm_c > 48 * 1024) {
    e = cudaFuncSetAttribute(kc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_c);
    if (e != cudaSuccess) return fail(std::string("column pass attribute: ") + cudaGetErrorString(e), VSAV_E_CUDA);
  }
  {
    const float2* in0 = reinterpret_cast<const float2*>(spec);
    const float2* in1 = nullptr;
    float a0 = 1.0f, a1 = 0.0f, oscale = 1.0f;
    int m = mult;
    double ms = 1.0;
    float2* o = scratch;
    const float2* t = tab;
    void* args[] = {(void*)&in0, (void*)&in1, (void*)&a0, (void*)&a1, (void*)&m, (void*)&ms,
                    (void*)&o, (void*)&oscale, (void*)&a, (void*)&t};
    e = cudaLaunchKernel(kc, dim3((unsigned)((long long)a.tiles * nf)), dim3(thr_c), args, sm_c, st);
    if (e != cudaSuccess) return fail(std::string("column pass launch: ") + cudaGetErrorString(e), VSAV_E_CUDA);
  }
  // row (x) pass: c2r of scratch rows (pitch nkx) -> out, scaled by 1/(Nx Ny)
  const int L = Nx / 2, logL = ilog2i(L);
  const long long nrows = (long long)nf * Ny;
  int nl = std::max(1, E * NT / L);
  while (nl > 1 && nl / 2 >= nrows) nl /= 2;
  const int thr_r = std::max(1, nl * L / E);
  const size_t sm_r = (size_t)(2 * nl * line_pitch(L) + nl) * sizeof(float2);
  const void* kr = (const void*)k_rows_c2r<float, E, NT>;
  if (sm_r > 48 * 1024) {
    e = cudaFuncSetAttribute(kr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_r);
    if (e != cudaSuccess) return fail(std::string("row pass attribute: ") + cudaGetErrorString(e), VSAV_E_CUDA);
  }
  {
    const float2* in = scratch;
    float* o = out;
    float scale = (float)(1.0 / ((double)Nx * Ny));
    int lL = logL, lnl = ilog2i(nl), kpv = nkx;
    long long nr = nrows;
    const float2* t = tab;
    void* args[] = {(void*)&in, (void*)&o, (void*)&scale, (void*)&lL, (void*)&lnl, (void*)&nr, (void*)&kpv, (void*)&t};
    e = cudaLaunchKernel(kr, dim3((unsigned)((nrows + nl - 1) / nl)), dim3(thr_r), args, sm_r, st);
    if (e != cudaSuccess) return fail(std::string("row pass launch: ") + cudaGetErrorString(e), VSAV_E_CUDA);
  }
  return VSAV_OK;
}

extern "C" const char* vsav_noalloc_error(void) { return g_noalloc_error.c_str(); }
