// khb_noalloc.cu -- khb_max_divb_noalloc: the divB diagnostic for callers that cannot allocate.
//
// Some callers cannot call cudaMalloc: a host framework that hands out device memory only from
// its own pre-reserved pool, or a diagnostic hook that holds only the field pointers and no
// khb_ctx (creating a context allocates its scratch).  This entry point needs no context and
// allocates nothing.  Its scratch -- one partial maximum per thread block -- is a file-scope
// __device__ array of KHB_NOALLOC_MAX_PARTIALS doubles (128 KiB) that every GPU which loads the
// library holds until the process exits.  Blocks with more corners than
// 256 * KHB_NOALLOC_MAX_PARTIALS are rejected.
//
// Host code may not pass the array's name to a kernel: on the host it is only a stand-in, not a
// device address.  The first call on each device therefore looks the address up with
// cudaGetSymbolAddress while that device is current, and keeps it for the life of the process
// (so that first call belongs before any stream capture, and a cudaDeviceReset, which unloads the
// module, ends its validity).  All calls share the one array and it keeps the last call's
// contents: every partial the reduction reads is written by the same call, so nothing needs
// clearing, but calls that overlap on the GPU (concurrent streams, or several host threads) race
// on it.
#include "khb_kernels.cuh"

#include <mutex>

#define KHB_NOALLOC_MAX_PARTIALS 16384
#define KHB_NOALLOC_MAX_DEVICES 64

namespace {

static __device__ __align__(256) double g_divb_partials[KHB_NOALLOC_MAX_PARTIALS];

std::mutex g_setup_mutex;
double* g_partials_addr[KHB_NOALLOC_MAX_DEVICES] = {nullptr};

thread_local std::string g_noalloc_err;

int noalloc_fail(int code, const std::string& msg)
{
    g_noalloc_err = msg;
    return code;
}

// Each block writes the maximum of its corners to partials[blockIdx.x]
__global__ void __launch_bounds__(256) k_divb_partials(khb::Dims d, khb::Phys ph, khb_fields U, int i_lo, int i_hi,
                                                       double* partials)
{
    const double m = khb::block_max256(khb::divb_of_thread(d, ph, U, i_lo, i_hi));
    if (threadIdx.x == 0) partials[blockIdx.x] = m;
}

// One block reduces the n partials into *out
__global__ void __launch_bounds__(256) k_max_partials(const double* partials, int n, double* out)
{
    double v = 0.;
    for (int x = threadIdx.x; x < n; x += 256) v = fmax(v, partials[x]);
    const double m = khb::block_max256(v);
    if (threadIdx.x == 0) *out = m;
}

} // namespace

extern "C" const char* khb_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

extern "C" int khb_max_divb_noalloc(const khb_config* cfg, const khb_fields* U, double* max_divb_out, void* stream)
{
    if (!cfg || !U || !max_divb_out) return noalloc_fail(KHB_ERR_ARG, "khb_max_divb_noalloc: NULL argument");
    khb::Dims d;
    khb::Phys ph;
    const char* why = nullptr;
    int rc = khb::derive_block(cfg, d, ph, &why);
    if (rc) return noalloc_fail(rc, why);
    cudaStream_t st = (cudaStream_t)stream;
    if (cfg->nvar < 8 || d.ndim < 2) {
        // no field, or no corners: 0, as khb_max_divb returns.  All-zero bytes are +0.0; the
        // memset is stream-ordered and the host does not wait for it.
        const cudaError_t e = cudaMemsetAsync(max_divb_out, 0, sizeof(double), st);
        return e == cudaSuccess ? KHB_OK : noalloc_fail(KHB_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
    }
    for (int v = 5; v < 8; ++v)
        if (!U->v[v]) return noalloc_fail(KHB_ERR_ARG, "khb_max_divb_noalloc: NULL B_U pointer");
    // same corner range as khb_max_divb (b_flux_ct.cpp:554-564)
    const int avoid_in = khb::phys_face(d.bc[0]), avoid_out = khb::phys_face(d.bc[1]);
    const int i_lo = d.is + avoid_in, i_hi = d.ie + !avoid_out;
    const long long corners = (long long)(i_hi - i_lo + 1)*(d.je - d.js + 2)*((d.ndim > 2) ? d.ke - d.ks + 2 : 1);
    const long long nblocks = (corners + 255) / 256;
    if (nblocks > KHB_NOALLOC_MAX_PARTIALS)
        return noalloc_fail(KHB_ERR_ARG, "khb_max_divb_noalloc: block has " + std::to_string(corners) +
                            " corners; the static scratch holds at most " +
                            std::to_string(256LL * KHB_NOALLOC_MAX_PARTIALS));
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(KHB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= KHB_NOALLOC_MAX_DEVICES) return noalloc_fail(KHB_ERR_ARG, "device ordinal out of range");
    double* partials = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        if (!g_partials_addr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_divb_partials);
            if (e != cudaSuccess)
                return noalloc_fail(KHB_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            g_partials_addr[dev] = (double*)p;
        }
        partials = g_partials_addr[dev];
    }
    k_divb_partials<<<(unsigned)nblocks, 256, 0, st>>>(d, ph, *U, i_lo, i_hi, partials);
    k_max_partials<<<1, 256, 0, st>>>(partials, (int)nblocks, max_divb_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return noalloc_fail(KHB_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return KHB_OK;
}
