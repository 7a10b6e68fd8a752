// necg_noalloc.cu -- the energy+gradient evaluation for callers that cannot
// allocate device memory.
//
// Some callers cannot call cudaMalloc at all: host programs that hand the whole
// GPU to their own memory pool at start-up and forbid any later allocation,
// code running where an allocation's implicit device synchronisation is not
// acceptable (a latency-bound loop between launches), or foreign-language hosts
// (a Fortran or C driver linking only this C ABI) that own no allocator for
// device memory.  necg_outprod_noalloc serves them: it runs the same kernels as
// necg_outprod, with every intermediate (per-basis and per-(l, P) records, H, S,
// the gradient-tile partials, row sums, status word) carved out of one fixed
// scratch array that this file defines at file scope.  The caller passes only
// x, f and g in device memory; the problem constants are host arrays.
//
// The scratch array is NECG_NOALLOC_SCRATCH_BYTES (32 MiB) on every GPU that
// loads this library, held until the process exits.  Every call uses the same
// array and leaves its contents behind; whatever must start at zero is cleared
// by the call itself.  Two calls that overlap on the GPU (different streams or
// host threads) race on the array; callers serialise them.  The array's device
// address is looked up once per device and kept for the life of the process, so
// a cudaDeviceReset (which unloads the library's module) must not be followed
// by further calls of this entry point.
#include <cuda_runtime.h>
#include <string.h>

#include <mutex>

#include "necg_kernels.cuh"
#include "necg_lanes.cuh"
#include "necg_math.cuh"
#include "../../include/necg.h"

#define NECG_NOALLOC_SCRATCH_BYTES (32u << 20)

static __device__ __align__(256) double necg_noalloc_scratch[NECG_NOALLOC_SCRATCH_BYTES / 8];

namespace {

constexpr int kMaxDevices = 64;
constexpr int kLcEnergy = 4;   // ket chunk of an energy tile
constexpr int kLcGrad = 16;    // ket chunk of a gradient tile (sets the partial-buffer depth)

std::mutex g_mutex;
double *g_scratch[kMaxDevices] = {};

// Device address of the scratch array on the current device.  The host-side
// symbol is only a stand-in; the address must come from cudaGetSymbolAddress,
// called once per device with that device current.
int scratch_address(double **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return NECG_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, necg_noalloc_scratch) != cudaSuccess || !p) return NECG_ERR_CUDA;
        g_scratch[dev] = (double *)p;
    }
    *out = g_scratch[dev];
    return NECG_OK;
}

size_t up32(size_t v) { return (v + 31) / 32 * 32; }  // 256-byte alignment in doubles

struct Carve {
    size_t bra, ket, part, H, S, rows, scal, status, tiles, sml, sms, scvv, total;
};

// Scratch layout in doubles for one call; total must fit the array.
Carve carve(int n, int nst, int K) {
    Carve c{};
    const size_t k = (size_t)K;
    const int nlc = (K + kLcGrad - 1) / kLcGrad;
    const int ntiles = necg::energy_tile_count(K, kLcEnergy);
    size_t off = 0;
    c.bra = off;    off = up32(off + (size_t)necg::bra_record_size(n) * k);
    c.ket = off;    off = up32(off + (size_t)necg::ket_record_size(n) * k * nst);
    c.part = off;   off = up32(off + (size_t)necg::part_stride(n) * k * nlc);
    c.H = off;      off = up32(off + k * k);
    c.S = off;      off = up32(off + k * k);
    c.rows = off;   off = up32(off + 2 * k);
    c.scal = off;   off = up32(off + 4);
    c.status = off; off = up32(off + 2);                  // 4 ints
    c.tiles = off;  off = up32(off + (size_t)ntiles);     // int2 = one double each
    c.sml = off;    off = up32(off + (size_t)nst * n * n);
    c.sms = off;    off = up32(off + (size_t)nst * 9 * n * n);
    c.scvv = off;   off = up32(off + (size_t)nst);
    c.total = off;
    return c;
}

// Energy tile list (the order of the handle path): thread per 32-row block kb
// writes its tiles (kb, 0 .. last / LC) after the tiles of all earlier blocks.
__global__ void noalloc_tiles_kernel(int2 *tiles, int K, int LC) {
    const int kb = blockIdx.x * blockDim.x + threadIdx.x;
    if (kb * 32 >= K) return;
    int start = 0;
    for (int b = 0; b < kb; ++b) {
        const int last = b * 32 + 31 < K - 1 ? b * 32 + 31 : K - 1;
        start += last / LC + 1;
    }
    const int last = kb * 32 + 31 < K - 1 ? kb * 32 + 31 : K - 1;
    for (int lc = 0; lc <= last / LC; ++lc) tiles[start + lc] = make_int2(kb, lc);
}

}  // namespace

extern "C" int necg_outprod_noalloc(int n, int nst, int K, double efs, const double *mass_host,
                                    const double *ncv_host, const double *scvv_host,
                                    const double *sml_host, const double *sms_host,
                                    const double *x_dev, double *f_dev, double *g_dev, void *stream) {
    if (n < 1 || n > 6) return NECG_ERR_UNSUPPORTED;
    if (nst < 1 || K < 1 || !mass_host || !ncv_host || !scvv_host || !sml_host || !sms_host || !x_dev ||
        !f_dev || !g_dev)
        return NECG_ERR_ARG;
    const Carve c = carve(n, nst, K);
    if (c.total * sizeof(double) > NECG_NOALLOC_SCRATCH_BYTES) return NECG_ERR_CAPACITY;
    double *base = nullptr;
    int rc = scratch_address(&base);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    int *status = (int *)(base + c.status);
    int2 *tiles = (int2 *)(base + c.tiles);
    // problem constants into the scratch array
    if (cudaMemcpyAsync(base + c.sml, sml_host, sizeof(double) * nst * n * n, cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(base + c.sms, sms_host, sizeof(double) * nst * 9 * n * n, cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(base + c.scvv, scvv_host, sizeof(double) * nst, cudaMemcpyHostToDevice, st))
        return NECG_ERR_CUDA;
    necg::launch_reset_status(status, st);
    const int nkb = (K + 31) / 32;
    noalloc_tiles_kernel<<<(nkb + 127) / 128, 128, 0, st>>>(tiles, K, kLcEnergy);

    necg::LaunchArgs a;
    memset(&a, 0, sizeof(a));
    a.n = n;
    a.K = K;
    a.nst = nst;
    a.efs = efs;
    a.mass_h = mass_host;
    a.ncv_h = ncv_host;
    const size_t siv = (size_t)K * (n * (n + 1) / 2 + 3 * n);
    a.iv = x_dev;
    a.C = x_dev + siv;
    a.sml = base + c.sml;
    a.sms = base + c.sms;
    a.scvv = base + c.scvv;
    a.bra = base + c.bra;
    a.ket = base + c.ket;
    a.tiles = tiles;
    a.ntiles = necg::energy_tile_count(K, kLcEnergy);
    a.LC_e = kLcEnergy;
    a.LC_g = kLcGrad;
    a.minb_e = 16;
    a.minb_g = 8;
    a.H = base + c.H;
    a.S = base + c.S;
    a.rows = base + c.rows;
    a.scal = base + c.scal;
    a.part = base + c.part;
    a.g = g_dev;
    a.status = status;
    a.lam = 1.0;
    if (necg::launch_prep(a, st) || necg::launch_energy(a, st)) return NECG_ERR_UNSUPPORTED;
    necg::launch_rows_finalize(a, f_dev, g_dev + siv, 0, 0.0, 0.0, st);
    if (necg::launch_grad(a, st)) return NECG_ERR_UNSUPPORTED;
    if (cudaGetLastError() != cudaSuccess) return NECG_ERR_CUDA;
    // synchronous: report the pair status of this evaluation
    int hs[2] = {0, 0};
    if (cudaMemcpyAsync(hs, status, sizeof(hs), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return NECG_ERR_CUDA;
    if (hs[0] & 1) return NECG_ERR_NOT_PD;
    if (hs[0] & 2) return NECG_ERR_NONFINITE;
    return NECG_OK;
}
