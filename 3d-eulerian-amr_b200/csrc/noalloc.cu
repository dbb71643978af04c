// amr_poisson_boundaries_noalloc: the domain-face potential computed with a
// scratch area that lives in the library image instead of one allocated at
// run time.
//
// Who needs it: a host code that hands all free device memory to its own
// pool allocator after start-up (so a later cudaMalloc fails or fragments
// that pool), or that calls in from a section where cudaMalloc/cudaFree are
// off limits because they can synchronise the device.  Such a caller sets the
// context up while allocation is still allowed (amr_create, the tree, one
// Poisson call) and afterwards recomputes the boundary potential through this
// entry point, which allocates nothing.
//
// The scratch is a file-scope device array of NOALLOC_SCRATCH_DOUBLES
// doubles (16 MiB).  Every GPU that loads this library holds it until the
// process exits, and every call shares it, so two calls that overlap on the
// GPU (on different streams or contexts) race on it.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "context.h"
#include "poisson.h"
#include "profiler.h"

namespace {

constexpr size_t NOALLOC_SCRATCH_DOUBLES = (size_t)1 << 21;  // 16 MiB
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

// Device address of g_noalloc_scratch per device.  In host code the array's
// name is only a host-side stand-in, so the address is looked up once per
// device, with that device current.
double* g_scratch_addr[NOALLOC_MAX_DEVICES] = {};
std::mutex g_scratch_mutex;

int scratch_for_current_device(amr_ctx* c, double** out) {
    int dev = -1, sdev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) {
        c->err = std::string("no usable current device: ") + cudaGetErrorString(e);
        return AMR_ERR_CUDA;
    }
    // the address below is the current device's copy of the array; the
    // kernels run on the context's stream, so the two devices must agree
    e = cudaStreamGetDevice(c->stream, &sdev);
    if (e != cudaSuccess) {
        c->err = std::string("cudaStreamGetDevice failed: ") + cudaGetErrorString(e);
        return AMR_ERR_CUDA;
    }
    if (sdev != dev) {
        c->err = "the context's device is not the current device";
        return AMR_ERR_STATE;
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            c->err = std::string("cudaGetSymbolAddress of the static scratch failed: ") + cudaGetErrorString(e);
            return AMR_ERR_CUDA;
        }
        g_scratch_addr[dev] = static_cast<double*>(p);
    }
    *out = g_scratch_addr[dev];
    return AMR_OK;
}

}  // namespace

extern "C" {

// Same result as amr_poisson_boundaries (source, octant monopoles, then the
// potential on every physical domain face), with the (subtree, point) partial
// sums kept in the static scratch.  The first call on a device looks up the
// scratch address (cudaGetSymbolAddress, which also loads the library's
// device code there); make that first call before any stream capture.
int amr_poisson_boundaries_noalloc(amr_ctx* c) {
    using namespace amr;
    if (!c) return AMR_ERR_ARG;
    if (!c->has_device) {
        c->err = "context has no device pool";
        return AMR_ERR_NODEVICE;
    }
    if (!has_gravity(c)) {
        c->err = "Poisson call on a context created without self-gravity";
        return AMR_ERR_ARG;
    }
    // the context's own Poisson buffers are allocated by the first ordinary
    // Poisson call; this entry point will not allocate them
    if (!c->d_bphi || !c->d_msrc || !c->d_allref || (c->n_bfaces > 0 && !c->d_pwalk)) {
        c->err = "Poisson buffers not set up: make one Poisson call (e.g. amr_poisson_set_source) first";
        return AMR_ERR_STATE;
    }
    // one point's partial sums (one per subtree) must fit; points are
    // batched through the scratch beyond that
    if ((size_t)c->n_pseg > NOALLOC_SCRATCH_DOUBLES) {
        c->err = "tree too large for the static scratch: " + std::to_string(c->n_pseg) +
                 " subtree sums per point, at most " + std::to_string(NOALLOC_SCRATCH_DOUBLES);
        return AMR_ERR_RANGE;
    }
    double* scratch = nullptr;
    {
        const int rc = scratch_for_current_device(c, &scratch);
        if (rc) return rc;
    }
    // every scratch entry that is read is written earlier in the same call,
    // so nothing has to be cleared between calls
    const int* order = c->d_slots + c->off_all[0];
    const int n = (int)c->all_slots.size();
    // the same profile classes as amr_poisson_boundaries (the scopes record
    // events only and count the launches; no device memory is allocated)
    {
        ProfScope ps_(c->prof, KC_SOURCE, c->stream);
        launch_set_source(c->geom, c->st, order, n, c->stream);
        launch_source_sums(c->geom, c->bt, c->st, order, n, c->d_msrc, c->d_allref, c->stream);
    }
    int rc;
    {
        ProfScope ps_(c->prof, KC_PHYS_BOUND, c->stream);
        rc = launch_phys_bound(c->geom, c->bt, c->d_bfaces, c->n_bfaces, order, phys_walk(c), c->d_msrc,
                               c->d_allref, c->d_bphi, scratch, NOALLOC_SCRATCH_DOUBLES, c->stream);
    }
    if (rc) {
        c->err = "static scratch too small for one point";
        return AMR_ERR_RANGE;
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        c->err = std::string("CUDA launch error: ") + cudaGetErrorString(e);
        return AMR_ERR_CUDA;
    }
    return AMR_OK;
}

}  // extern "C"
