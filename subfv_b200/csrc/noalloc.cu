// subfv_compute_dt_noalloc: the CFL time-step reduction of compute_dt for callers that
// cannot allocate device memory at call time.
//
// Who needs it: a host code that reserves all of its device memory when it starts and
// is forbidden to allocate afterwards (a memory-capped job sharing the GPU, a solver
// embedded in a larger application that owns the allocator), or a caller stepping inside
// a region where cudaMalloc is not allowed. Such a caller hands in device buffers it
// already owns (sol, vp, the dt output) and a mesh it created at start-up; this entry
// point then calls no cudaMalloc, cudaFree or any allocating routine.
//
// Its only scratch is g_dt_partial below: one minimum per thread block, at most
// kNoAllocMaxBlocks blocks of kNoAllocBlock cells, so meshes of up to
// kNoAllocMaxBlocks * kNoAllocBlock = 4,194,304 cells; larger meshes are rejected. The
// array is part of the loaded library: every GPU that loads it holds these 128 KiB
// until the process exits. Every call writes each slot it later reads, so nothing
// needs clearing between calls; but all calls share the one array, so two calls whose
// work overlaps on the GPU (different streams, or one device used from two threads)
// race on it and must not be issued concurrently.
//
// The kernels run on the mesh's stream, which does not wait for the caller's streams:
// d_sol and d_vp must be complete (the stream that wrote them synchronised) before the
// call. The scratch address is looked up on the device that holds the mesh, whichever
// device is current, and the caller's current device is restored afterwards.
//
// The arithmetic is that of k_lag_cell's CFL terms (lagrange_module.F90:240-283),
// including the non-finite check that sets the mesh's status word, so the result and
// the status equal subfv_compute_dt's bit for bit.
#include <mutex>

#include "../../include/subfv.h"
#include "common.cuh"
#include "mesh_dev.cuh"

namespace subfv {
namespace {

constexpr int kNoAllocBlock = 256;
constexpr int kNoAllocMaxBlocks = 16384;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_dt_partial[kNoAllocMaxBlocks];

// Device address of g_dt_partial per device. The host symbol is only a handle: a kernel
// given its host address would fault (or read host memory), so the address is looked up
// once per device with that device current.
std::mutex g_mu;
double* g_addr[kMaxDevices] = {};

__device__ inline double warp_min_na(double x) {
  for (int o = 16; o > 0; o >>= 1) x = fmin(x, __shfl_xor_sync(0xffffffffu, x, o));
  return x;
}

__global__ void __launch_bounds__(kNoAllocBlock) k_dt_partial(DevMesh m, const double* __restrict__ sol5,
                                                              const double* __restrict__ vp3, double* partial) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  double dtloc = 1e6;  // compute_dt starts from dt = 1e6
  if (c < m.ne) {
    const double* u = sol5 + 5 * (size_t)c;
    double pme = lag_pressure(u[0], u[1], u[2], u[3], u[4]);
    double csnd = sqrt(kGamma * pme * u[0]);
    const double vse_c = m.vol_se[c < m.nse ? c : 0];  // sub_elem(i) with i the cell (reference quirk)
    bool bad = false;
    for (int q = m.csf_off[c]; q < m.csf_off[c + 1]; ++q) {
      int e = m.csf[q];
      int p = e >> 1, side = e & 1;
      int sf = m.vsf_identity ? p : m.vsf[p];
      int f = m.sf_face[sf];
      double4 fn = m.fn[f];
      double area = m.sfa[sf];
      int sv = m.sf_vert[sf];
      int2 se = m.sf_se[sf];
      int sub = side == 0 ? se.x : se.y;
      double sg = side == 0 ? 1.0 : -1.0;
      const double* vps = vp3 + 3 * (size_t)sv;
      double t1 = vse_c / (area * csnd);
      if (t1 < dtloc) dtloc = t1;
      bad = bad || !(t1 >= 0.0);
      if (sub >= 0) {
        double vn = dot3(vps[0], vps[1], vps[2], sg * fn.x, sg * fn.y, sg * fn.z);
        double t2 = 0.8 * m.vol_se[sub] / (1e-8 + fabs(vn) * fn.w);
        if (t2 < dtloc) dtloc = t2;
        bad = bad || !(t2 >= 0.0);
      }
    }
    if (bad) atomicOr(m.status, kErrNonFinite);
  }
  __shared__ double wmin[kNoAllocBlock / 32];
  double x = warp_min_na(dtloc);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) wmin[wid] = x;
  __syncthreads();
  if (wid == 0) {
    x = lane < kNoAllocBlock / 32 ? wmin[lane] : 1e6;
    x = warp_min_na(x);
    if (lane == 0) partial[blockIdx.x] = x;
  }
}

__global__ void __launch_bounds__(kNoAllocBlock) k_dt_final(const double* partial, int nblocks, double cfl,
                                                            double* dt_out) {
  double x = 1e6;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) x = fmin(x, partial[i]);
  __shared__ double wmin[kNoAllocBlock / 32];
  x = warp_min_na(x);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) wmin[wid] = x;
  __syncthreads();
  if (wid == 0) {
    x = lane < kNoAllocBlock / 32 ? wmin[lane] : 1e6;
    x = warp_min_na(x);
    if (lane == 0) *dt_out = cfl * x;
  }
}

}  // namespace

const DevMesh& mesh_device_view(const subfv_mesh* m);

}  // namespace subfv

using namespace subfv;

extern "C" int subfv_compute_dt_noalloc(subfv_mesh* mesh, const double* d_sol, const double* d_vp, double cfl,
                                        double* d_dt) {
  if (!mesh || !d_sol || !d_vp || !d_dt) {
    set_error("subfv_compute_dt_noalloc: null argument");
    return -2;
  }
  const DevMesh& m = mesh_device_view(mesh);
  const int nblocks = (m.ne + kNoAllocBlock - 1) / kNoAllocBlock;
  if (nblocks > kNoAllocMaxBlocks) {
    set_error("subfv_compute_dt_noalloc: mesh has more than 4,194,304 cells (the static scratch holds 16,384 "
              "block minima of 256 cells); use subfv_compute_dt");
    return -4;
  }
  // the device that holds the mesh (its status word lives there)
  cudaPointerAttributes attr{};
  SUBFV_CUDA(cudaPointerGetAttributes(&attr, m.status));
  const int dev = attr.device;
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("subfv_compute_dt_noalloc: device index out of range");
    return -2;
  }
  int cur = 0;
  SUBFV_CUDA(cudaGetDevice(&cur));
  if (cur != dev) SUBFV_CUDA(cudaSetDevice(dev));
  struct Restore {
    int cur, dev;
    ~Restore() {
      if (cur != dev) cudaSetDevice(cur);
    }
  } restore{cur, dev};
  double* partial = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {  // first call on this device: look up the array's device address
      void* p = nullptr;
      SUBFV_CUDA(cudaGetSymbolAddress(&p, g_dt_partial));
      g_addr[dev] = static_cast<double*>(p);
    }
    partial = g_addr[dev];
  }
  SUBFV_CUDA(cudaMemsetAsync(m.status, 0, sizeof(unsigned), m.stream));
  k_dt_partial<<<nblocks, kNoAllocBlock, 0, m.stream>>>(m, d_sol, d_vp, partial);
  k_dt_final<<<1, kNoAllocBlock, 0, m.stream>>>(partial, nblocks, cfl, d_dt);
  SUBFV_CUDA(cudaGetLastError());
  unsigned st = 0;
  SUBFV_CUDA(cudaMemcpyAsync(&st, m.status, sizeof(unsigned), cudaMemcpyDeviceToHost, m.stream));
  SUBFV_CUDA(cudaStreamSynchronize(m.stream));
  return (int)st;
}
