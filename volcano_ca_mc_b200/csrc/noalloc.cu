// noalloc.cu -- vca_mc_energy_noalloc: the Potts energy of a spin grid that lives in the caller's
// device memory, computed without allocating anything.
//
// It restates the reduction of vca_mc_energy (PottsMC::totalEnergy, engine/src/mc/PottsMC.cpp:590-664)
// for callers that own every byte of device memory: the per-block partial sums and the
// last-block ticket live in one file-scope __device__ array of fixed size, whose address host code
// looks up with cudaGetSymbolAddress (on every call outside stream capture, so that a context that
// was torn down and made again -- cudaDeviceReset -- never leaves a stale address behind).  The
// result is written to a device double of the caller, on the caller's stream.
#include <cuda_runtime.h>

#include <mutex>

#include "vca_device.cuh"
#include "vca_internal.h"

namespace vca {
namespace {

constexpr int kNaThreads = 256;
constexpr int kNaCellsPerThread = 16;
constexpr uint64_t kNaCellsPerBlock = (uint64_t)kNaThreads * kNaCellsPerThread;  // 4096
constexpr int kNaMaxBlocks = 65536;
// Largest grid: 65536 blocks x 4096 cells = 2^28 cells (e.g. 1024 x 1024 x 256).
constexpr uint64_t kNaMaxCells = (uint64_t)kNaMaxBlocks * kNaCellsPerBlock;
constexpr int kNaTicket = kNaMaxBlocks;  // index of the last-block ticket in the scratch array
constexpr int kNaMaxDevices = 64;

// Scratch: one partial sum per block (512 KiB) and the ticket, 256-byte aligned.
static __device__ __align__(256) unsigned long long g_energy_scratch[kNaMaxBlocks + 32];

struct NaGrid {
    int nx, ny, nz;
    int per[3];
    int forward;        // deterministic neighbourhood: forward half of the offsets, each pair once
    int variants;
    FastMod var_mod;
    uint64_t prefix;    // hashPrefix(seed, mcs): neighbourhood variant of the cell at MCS mcs
    uint64_t n;
    int blocks;
    double scale;       // J (forward pairs) or J / 2 (sum of per-cell energies)
};

__device__ __forceinline__ bool na_wrap(int& v, int n, int periodic) {
    if (v >= 0 && v < n) return true;
    if (!periodic || n == 1) return false;
    v = v < 0 ? v + n : v - n;
    return true;
}

__device__ __forceinline__ unsigned long long na_block_sum(unsigned long long v, unsigned long long* s_warp) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, off);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) s_warp[warp] = v;
    __syncthreads();
    unsigned long long total = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kNaThreads / 32; ++w) total += s_warp[w];
    return total;  // valid in thread 0
}

// One block per 4096 cells: unlike in-domain neighbours of every in-domain cell (spin != 0), the
// block's sum into scratch[block]; the block that takes the last ticket adds the partials in block
// order, writes scale * sum to *energy and puts the ticket back to zero.
__global__ __launch_bounds__(kNaThreads) void mc_energy_noalloc_kernel(NaGrid g, NbTable nb, const int32_t* spin,
                                                                      unsigned long long* scratch, double* energy) {
    __shared__ unsigned long long s_warp[kNaThreads / 32];
    __shared__ bool s_last;
    const uint64_t base = (uint64_t)blockIdx.x * kNaCellsPerBlock;
    unsigned long long mine = 0;
    for (int i = 0; i < kNaCellsPerThread; ++i) {
        const uint64_t c = base + (uint64_t)i * kNaThreads + threadIdx.x;
        if (c >= g.n) break;
        const int32_t s = spin[c];
        if (s == 0) continue;
        const uint32_t cc = (uint32_t)c;  // n <= 2^28
        const uint32_t r = cc / (uint32_t)g.nx;
        const int x = (int)(cc - r * (uint32_t)g.nx);
        const int y = (int)(r % (uint32_t)g.ny);
        const int z = (int)(r / (uint32_t)g.ny);
        int var = 0;
        if (!g.forward && g.variants > 1) var = (int)fast_mod(hash_salt(hash_index(g.prefix, c), kSaltNeighborhood), g.var_mod);
        int in_dom = 0, same = 0;
        for (int k = 0; k < nb.count[var]; ++k) {
            const int dx = nb.off[var][k][0], dy = nb.off[var][k][1], dz = nb.off[var][k][2];
            if (g.forward && !(dz > 0 || (dz == 0 && (dy > 0 || (dy == 0 && dx > 0))))) continue;
            int qx = x + dx, qy = y + dy, qz = z + dz;
            if (!na_wrap(qx, g.nx, g.per[0]) || !na_wrap(qy, g.ny, g.per[1]) || !na_wrap(qz, g.nz, g.per[2])) continue;
            const int32_t t = spin[(uint64_t)qx + (uint64_t)g.nx * ((uint64_t)qy + (uint64_t)g.ny * qz)];
            in_dom += t != 0;
            same += t == s;
        }
        mine += (unsigned long long)(in_dom - same);
    }
    const unsigned long long block = na_block_sum(mine, s_warp);
    if (threadIdx.x == 0) {
        scratch[blockIdx.x] = block;
        __threadfence();
        const unsigned long long ticket = atomicAdd(&scratch[kNaTicket], 1ULL);
        s_last = ticket == (unsigned long long)(g.blocks - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    unsigned long long part = 0;
    for (int b = threadIdx.x; b < g.blocks; b += kNaThreads) part += __ldcg(&scratch[b]);
    __syncthreads();  // s_warp is reused
    const unsigned long long total = na_block_sum(part, s_warp);
    if (threadIdx.x == 0) {
        *energy = g.scale * (double)total;
        scratch[kNaTicket] = 0;
    }
}

std::mutex g_na_mutex;
unsigned long long* g_na_scratch[kNaMaxDevices] = {};

// Address of the scratch array on the current device.  Outside stream capture it is looked up on
// every call (the address belongs to the device's current context; a reset context gets a new one)
// and remembered; during capture, where a lookup could load the module and break the capture, the
// remembered address of the last call outside capture is used, and a device that never had one is
// refused.
vca_status na_scratch(int device, bool capturing, unsigned long long** out) {
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (capturing) {
        if (!g_na_scratch[device]) {
            set_error("vca_mc_energy_noalloc: the first call on a device must come before any stream capture "
                      "(it looks up the address of the static scratch)");
            return VCA_ERR_STATE;
        }
        *out = g_na_scratch[device];
        return VCA_OK;
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_energy_scratch);
    if (e != cudaSuccess) {
        set_error(std::string("vca_mc_energy_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return VCA_ERR_CUDA;
    }
    g_na_scratch[device] = static_cast<unsigned long long*>(p);
    *out = g_na_scratch[device];
    return VCA_OK;
}

vca_status na_device_pointer(const void* p, int device, const char* what) {
    cudaPointerAttributes attr{};
    const cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error(std::string("vca_mc_energy_noalloc: ") + what + " is not a CUDA pointer: " + cudaGetErrorString(e));
        return VCA_ERR_ARG;
    }
    if ((attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) || attr.device != device) {
        set_error(std::string("vca_mc_energy_noalloc: ") + what + " must be device (or managed) memory of the current device " +
                  std::to_string(device));
        return VCA_ERR_ARG;
    }
    return VCA_OK;
}

}  // namespace
}  // namespace vca

using namespace vca;

extern "C" {

vca_status vca_mc_energy_noalloc(const int32_t* spins, int nx, int ny, int nz, int neighborhood, int boundary,
                                 int domain_full, uint64_t seed, int mcs, double J, double* energy, void* stream) {
    if (nx < 1 || ny < 1 || nz < 1 || mcs < 0 || (boundary != VCA_BC_ABSORBING && boundary != VCA_BC_PERIODIC)) {
        set_error("vca_mc_energy_noalloc: invalid dimensions, boundary or mcs");
        return VCA_ERR_ARG;
    }
    const uint64_t n = (uint64_t)nx * (uint64_t)ny * (uint64_t)nz;
    if (n > kNaMaxCells) {
        set_error("vca_mc_energy_noalloc: " + std::to_string(n) + " cells exceed the fixed scratch of this entry point (at most " +
                  std::to_string(kNaMaxCells) + " cells = 65536 blocks of 4096); use vca_mc_energy for larger grids");
        return VCA_ERR_ARG;
    }
    if (!spins || !energy) {
        set_error("vca_mc_energy_noalloc: null spins or energy pointer");
        return VCA_ERR_ARG;
    }
    NbTable nb;
    if (neighborhood < VCA_NB_VON_NEUMANN || neighborhood > VCA_NB_HEXAGONAL || !build_nb(neighborhood, nx, ny, nz, nb)) {
        set_error("vca_mc_energy_noalloc: the neighbourhood does not exist for these dimensions "
                  "(hexagonal is 2D only; a grid needs two axes of size > 1)");
        return VCA_ERR_ARG;
    }
    int device = 0;
    VCA_CUDA(cudaGetDevice(&device));
    if (device < 0 || device >= kNaMaxDevices) {
        set_error("vca_mc_energy_noalloc: device ordinal out of range");
        return VCA_ERR_ARG;
    }
    if (vca_status s = na_device_pointer(spins, device, "spins")) return s;
    if (vca_status s = na_device_pointer(energy, device, "energy")) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (st != nullptr && st != cudaStreamLegacy && st != cudaStreamPerThread) {
        int stream_device = -1;
        VCA_CUDA(cudaStreamGetDevice(st, &stream_device));
        if (stream_device != device) {
            set_error("vca_mc_energy_noalloc: the stream belongs to device " + std::to_string(stream_device) +
                      ", not to the current device " + std::to_string(device));
            return VCA_ERR_ARG;
        }
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    VCA_CUDA(cudaStreamIsCapturing(st, &cap));
    unsigned long long* scratch = nullptr;
    if (vca_status s = na_scratch(device, cap != cudaStreamCaptureStatusNone, &scratch)) return s;

    const bool periodic = boundary == VCA_BC_PERIODIC;
    NaGrid g{};
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.per[0] = periodic && nx > 1;
    g.per[1] = periodic && ny > 1;
    g.per[2] = periodic && domain_full && nz > 1;  // the basalt domain has no periodic z (PottsMC.cpp:18)
    g.forward = nb.variants == 1;
    g.variants = nb.variants;
    g.var_mod = make_fastmod((uint64_t)nb.variants);
    g.prefix = hash_prefix(seed, (uint64_t)mcs);
    g.n = n;
    g.blocks = (int)((n + kNaCellsPerBlock - 1) / kNaCellsPerBlock);
    g.scale = g.forward ? J : 0.5 * J;
    // the ticket must start at zero: the kernel's last block puts it back, this makes every call
    // independent of an earlier one that did not finish
    VCA_CUDA(cudaMemsetAsync(scratch + kNaTicket, 0, sizeof(unsigned long long), st));
    mc_energy_noalloc_kernel<<<g.blocks, kNaThreads, 0, st>>>(g, nb, spins, scratch, energy);
    VCA_CUDA(cudaGetLastError());
    return VCA_OK;
}

}  // extern "C"
