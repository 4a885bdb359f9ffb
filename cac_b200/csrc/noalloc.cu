// Per-replica potential energy without any device allocation.
//
// Some callers cannot allocate device memory: a host program that runs inside
// another framework's memory pool (which has reserved the GPU's memory up
// front and must stay the only allocator), or a serving loop whose other
// streams must not be stalled, since cudaFree waits for the whole device.
// This entry point is the same reduction as cacb200_replica_energy, but
// its device scratch (the per-replica table of offsets and counts, and the
// per-replica sums) lives in one fixed array of this file, set up once per
// device, instead of buffers a context allocates.
#include <cstdio>
#include <vector>

#include "../../include/cacb200.h"
#include "ctx.cuh"
#include "device.cuh"

namespace cacb200 {
namespace {

// Scratch for at most NOALLOC_MAX_REPLICAS replicas (96 KiB); every GPU that
// loads the library holds it until the process exits.
constexpr int NOALLOC_MAX_REPLICAS = CACB200_NOALLOC_MAX_REPLICAS;
struct NoAllocScratch {
  int meta[4 * NOALLOC_MAX_REPLICAS];  // per replica r: atom offset, atom count, element offset, element count
                                       // at 4r .. 4r+3 (a call copies only its replicas' 16 bytes each)
  double sum[NOALLOC_MAX_REPLICAS];    // energy of each replica
};
static __device__ __align__(256) NoAllocScratch noalloc_scratch;

// One block per replica: atoms' own energies plus node energies times the
// node weight, summed in a fixed order (the kernel of cacb200_replica_energy
// with its table and results in the fixed scratch).
__global__ void k_replica_energy_fixed(const double *eatom, const double *enode, double node_weight,
                                       NoAllocScratch *sc) {
  const int r = blockIdx.x;
  const int *m = sc->meta + 4 * r;
  const int aoff = m[0], na = m[1], eoff = m[2], ne = m[3];
  double s = 0.0;
  for (int i = threadIdx.x; i < na; i += blockDim.x) s += eatom[aoff + i];
  double t = 0.0;
  for (int k = threadIdx.x; k < 8 * ne; k += blockDim.x) t += enode[8 * (size_t)eoff + k];
  double v[1] = {s + node_weight * t};
  block_reduce_store<1>(v, sc->sum);   // sum[r] for block r: every used slot is overwritten
}

// Device address of the scratch on the current device, looked up on every
// call (a few microseconds): a cached address would dangle after a device
// reset reloads the module.  In host code `noalloc_scratch` only names a
// host-side stand-in.
constexpr int MAX_DEVICES = 64;

cudaError_t scratch_for(NoAllocScratch **out) {
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, noalloc_scratch);
  if (e != cudaSuccess) return e;
  *out = static_cast<NoAllocScratch *>(p);
  return cudaSuccess;
}

}  // namespace
}  // namespace cacb200

namespace {
// the calling thread's last failure of cacb200_replica_energy_noalloc
thread_local char noalloc_error[160] = "";

int noalloc_fail(int code, const char *what) {
  std::snprintf(noalloc_error, sizeof noalloc_error, "cacb200_replica_energy_noalloc: %s", what);
  return code;
}
}  // namespace

extern "C" const char *cacb200_noalloc_last_error(void) { return noalloc_error; }

extern "C" int cacb200_replica_energy_noalloc(int device, const double *eatom, const double *enode,
                                              int nreplicas, const int *natoms, const int *nelements,
                                              double node_weight, double *energy, void *stream) {
  using namespace cacb200;
  if (nreplicas < 1 || nreplicas > NOALLOC_MAX_REPLICAS) {
    char m[120];
    std::snprintf(m, sizeof m, "%d replicas; the fixed scratch holds 1 to %d", nreplicas, NOALLOC_MAX_REPLICAS);
    return noalloc_fail(CACB200_EINVAL, m);
  }
  if (!natoms || !nelements || !energy) return noalloc_fail(CACB200_EINVAL, "null count or output array");
  if (device < 0 || device >= MAX_DEVICES) return noalloc_fail(CACB200_EINVAL, "device index out of range");
  std::vector<int> meta(4 * (size_t)nreplicas, 0);
  long a = 0, e = 0;
  for (int r = 0; r < nreplicas; r++) {
    if (natoms[r] < 0 || nelements[r] < 0) return noalloc_fail(CACB200_EINVAL, "negative site count");
    meta[4 * r] = (int)a;
    meta[4 * r + 1] = natoms[r];
    meta[4 * r + 2] = (int)e;
    meta[4 * r + 3] = nelements[r];
    a += natoms[r];
    e += nelements[r];
  }
  if (a >= (1L << 31) || 8 * e >= (1L << 31)) return noalloc_fail(CACB200_EINVAL, "more than 2^31 sites");
  if ((a > 0 && !eatom) || (e > 0 && !enode)) return noalloc_fail(CACB200_EINVAL, "null per-site energy array");
  int prev = 0;
  if (cudaGetDevice(&prev) != cudaSuccess) return noalloc_fail(CACB200_ECUDA, "cudaGetDevice failed");
  if (cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(CACB200_ECUDA, "cudaSetDevice failed");
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  NoAllocScratch *sc = nullptr;
  cudaError_t err = scratch_for(&sc);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(sc->meta, meta.data(), sizeof(int) * meta.size(), cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) {
    k_replica_energy_fixed<<<nreplicas, 256, 0, st>>>(eatom, enode, node_weight, sc);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(energy, sc->sum, sizeof(double) * nreplicas, cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  cudaSetDevice(prev);
  if (err != cudaSuccess) {
    cudaGetLastError();
    return noalloc_fail(CACB200_ECUDA, cudaGetErrorString(err));
  }
  noalloc_error[0] = '\0';
  return CACB200_OK;
}
