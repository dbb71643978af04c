// Helmholtz EOS host side: table reading, device upload, C ABI
// (include/helm_b200.h).
#include <cuda_runtime.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "helm_internal.h"

using namespace amr;

struct helm_ctx {
    std::string err;
    double* d_node = nullptr;
    double* d_tj = nullptr;
    double* d_di = nullptr;
    HelmTable tab{};
    // staging of the host-array calls: inputs, outputs, statuses
    double* d_stage = nullptr;
    size_t stage_cap = 0;  // doubles
    cudaStream_t stream = nullptr;
};

namespace {

#define HCUDA(call)                                                                             \
    do {                                                                                        \
        cudaError_t e__ = (call);                                                               \
        if (e__ != cudaSuccess) {                                                               \
            c->err = std::string("CUDA error: ") + cudaGetErrorString(e__) + " at " + #call;   \
            return AMR_ERR_CUDA;                                                                \
        }                                                                                       \
    } while (0)

// helmholtz_set_cgs_units + eos_from_code factors (helmeos.cpp:132-162)
HelmUnits make_units(double cm, double g, double s, double K) {
    const double erg = g * cm * cm / s / s;
    const double dyne = g * cm / s / s;
    HelmUnits u;
    u.f_p = dyne / std::pow(cm, 2);
    u.f_e = erg / g;
    u.f_T = K;
    u.f_cs = cm / s;
    u.f_cv = erg / g / K;
    u.f_rho = g / std::pow(cm, 3);
    u.f_s = erg / K / g;
    u.f_dsdt = erg / K / K / g;
    return u;
}

int read_table(helm_ctx* c, const char* path, std::vector<double>& node) {
    FILE* fp = fopen(path, "rb");
    if (!fp) {
        c->err = std::string("cannot open Helmholtz table ") + path;
        return AMR_ERR_ARG;
    }
    std::vector<char> buf;
    {
        char chunk[1 << 16];
        size_t k;
        while ((k = fread(chunk, 1, sizeof(chunk), fp)) > 0) buf.insert(buf.end(), chunk, chunk + k);
    }
    fclose(fp);
    buf.push_back('\0');
    const size_t want = (size_t)HELM_IMAX * HELM_JMAX * 9;
    node.assign((size_t)HELM_IMAX * HELM_JMAX * HELM_NODE, 0.0);
    const char* p = buf.data();
    for (size_t q = 0; q < want; q++) {
        char* end = nullptr;
        errno = 0;
        const double v = strtod(p, &end);
        if (end == p) {
            c->err = "Helmholtz table " + std::string(path) + ": expected " + std::to_string(want) +
                     " numbers, found " + std::to_string(q);
            return AMR_ERR_ARG;
        }
        p = end;
        // file order: node (i inner, j outer), 9 values per node
        node[(q / 9) * HELM_NODE + q % 9] = v;
    }
    return AMR_OK;
}

int ensure_stage(helm_ctx* c, size_t doubles) {
    if (doubles <= c->stage_cap) return AMR_OK;
    if (c->d_stage) cudaFree(c->d_stage);
    c->d_stage = nullptr;
    c->stage_cap = 0;
    HCUDA(cudaMalloc(&c->d_stage, sizeof(double) * doubles));
    c->stage_cap = doubles;
    return AMR_OK;
}

int first_error(const int* status, long long n) {
    int worst = AMR_OK;
    for (long long q = 0; q < n; q++) {
        if (status[q] == 4) worst = AMR_ERR_NOCONVERGE;
        else if (status[q] != 0) return AMR_ERR_RANGE;
    }
    return worst;
}

}  // namespace

extern "C" {

int helm_create(const char* path, helm_ctx** out) {
    if (!path || !out) return AMR_ERR_ARG;
    *out = nullptr;
    helm_ctx* c = new helm_ctx;
    std::vector<double> node;
    int rc = read_table(c, path, node);
    if (rc) {
        fprintf(stderr, "[helm] %s\n", c->err.c_str());
        delete c;
        return rc;
    }
    // read_helm_table (helmeos.cpp:73-130): node positions and interval
    // tables, computed on the host with the C library's pow exactly as the
    // reference does
    const double tlo = 3.0, thi = 13.0, dlo = -12.0, dhi = 15.0;
    const double tstp = (thi - tlo) / double(HELM_JMAX - 1);
    const double dstp = (dhi - dlo) / double(HELM_IMAX - 1);
    std::vector<double> t(HELM_JMAX), d(HELM_IMAX), tj((size_t)HELM_JMAX * 8, 0.0), di((size_t)HELM_IMAX * 8, 0.0);
    for (int j = 0; j < HELM_JMAX; j++) t[j] = std::pow(10.0, tlo + j * tstp);
    for (int i = 0; i < HELM_IMAX; i++) d[i] = std::pow(10.0, dlo + i * dstp);
    for (int j = 0; j < HELM_JMAX; j++) {
        tj[8 * j] = t[j];
        if (j < HELM_JMAX - 1) {
            const double dth = t[j + 1] - t[j];
            const double dt2 = dth * dth;
            tj[8 * j + 1] = dth;
            tj[8 * j + 2] = dt2;
            tj[8 * j + 3] = 1.0 / dth;
            tj[8 * j + 4] = 1.0 / dt2;
        }
    }
    for (int i = 0; i < HELM_IMAX; i++) {
        di[8 * i] = d[i];
        if (i < HELM_IMAX - 1) {
            const double dd = d[i + 1] - d[i];
            const double dd2 = dd * dd;
            di[8 * i + 1] = dd;
            di[8 * i + 2] = dd2;
            di[8 * i + 3] = 1.0 / dd;
            di[8 * i + 4] = 1.0 / dd2;
        }
    }
    auto fail = [&](cudaError_t e, const char* what) {
        c->err = std::string("CUDA error: ") + cudaGetErrorString(e) + " at " + what;
        fprintf(stderr, "[helm] %s\n", c->err.c_str());
        helm_destroy(c);
        return AMR_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    if ((e = cudaMalloc(&c->d_node, sizeof(double) * node.size())) != cudaSuccess) return fail(e, "node");
    if ((e = cudaMalloc(&c->d_tj, sizeof(double) * tj.size())) != cudaSuccess) return fail(e, "tj");
    if ((e = cudaMalloc(&c->d_di, sizeof(double) * di.size())) != cudaSuccess) return fail(e, "di");
    if ((e = cudaMemcpy(c->d_node, node.data(), sizeof(double) * node.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e, "node upload");
    if ((e = cudaMemcpy(c->d_tj, tj.data(), sizeof(double) * tj.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e, "tj upload");
    if ((e = cudaMemcpy(c->d_di, di.data(), sizeof(double) * di.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(e, "di upload");
    HelmTable& H = c->tab;
    H.node = c->d_node;
    H.tj = c->d_tj;
    H.di = c->d_di;
    H.tlo = tlo;
    H.tstpi = 1.0 / tstp;
    H.dlo = dlo;
    H.dstpi = 1.0 / dstp;
    H.t_first = t[0];
    H.t_last = t[HELM_JMAX - 1];
    H.d_first = d[0];
    H.d_last = d[HELM_IMAX - 1];
    H.u = make_units(1.0, 1.0, 1.0, 1.0);
    *out = c;
    return AMR_OK;
}

void helm_destroy(helm_ctx* c) {
    if (!c) return;
    if (c->stream) cudaStreamSynchronize(c->stream);
    if (c->d_node) cudaFree(c->d_node);
    if (c->d_tj) cudaFree(c->d_tj);
    if (c->d_di) cudaFree(c->d_di);
    if (c->d_stage) cudaFree(c->d_stage);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char* helm_last_error(helm_ctx* c) { return c ? c->err.c_str() : "null Helmholtz context"; }

int helm_set_cgs_units(helm_ctx* c, double cm, double g, double s, double K) {
    if (!c || !(cm > 0) || !(g > 0) || !(s > 0) || !(K > 0)) return AMR_ERR_ARG;
    c->tab.u = make_units(cm, g, s, K);
    return AMR_OK;
}

int helm_eos_device(helm_ctx* c, long long n, const double* rho, const double* T, const double* abar,
                    const double* zbar, double* p, double* e, double* cs, double* cv, double* s, double* dsdt,
                    int* status, void* stream) {
    if (!c || n < 0 || (n > 0 && (!rho || !T || !abar || !zbar || !status))) return AMR_ERR_ARG;
    launch_helm_eos(c->tab, n, rho, T, abar, zbar, p, e, cs, cv, s, dsdt, status, (cudaStream_t)stream);
    HCUDA(cudaGetLastError());
    return AMR_OK;
}

int helm_invert_T_device(helm_ctx* c, long long n, const double* rho, const double* target, const double* abar,
                         const double* zbar, int from_entropy, double* T, double* p, double* e, double* cs,
                         double* cv, double* s, int* iters, int* status, void* stream) {
    if (!c || n < 0 || (n > 0 && (!rho || !target || !abar || !zbar || !T || !status))) return AMR_ERR_ARG;
    launch_helm_invert(c->tab, n, rho, target, abar, zbar, from_entropy ? 1 : 0, T, p, e, cs, cv, s, iters, status,
                       (cudaStream_t)stream);
    HCUDA(cudaGetLastError());
    return AMR_OK;
}

int helm_eos_batch(helm_ctx* c, long long n, const double* rho, const double* T, const double* abar,
                   const double* zbar, double* p, double* e, double* cs, double* cv, double* s, double* dsdt,
                   int* status) {
    if (!c || n < 0 || (n > 0 && (!rho || !T || !abar || !zbar))) return AMR_ERR_ARG;
    if (n == 0) return AMR_OK;
    const size_t N = (size_t)n;
    // layout: 4 inputs, 6 outputs, statuses (as int, rounded up to doubles)
    const size_t st_d = (N * sizeof(int) + sizeof(double) - 1) / sizeof(double);
    if (int rc = ensure_stage(c, 10 * N + st_d)) return rc;
    double* D = c->d_stage;
    const double* ins[4] = {rho, T, abar, zbar};
    for (int k = 0; k < 4; k++)
        HCUDA(cudaMemcpyAsync(D + k * N, ins[k], sizeof(double) * N, cudaMemcpyHostToDevice, c->stream));
    double* outs[6] = {p, e, cs, cv, s, dsdt};
    double* dout[6];
    for (int k = 0; k < 6; k++) dout[k] = outs[k] ? D + (4 + k) * N : nullptr;
    int* dst = reinterpret_cast<int*>(D + 10 * N);
    launch_helm_eos(c->tab, n, D, D + N, D + 2 * N, D + 3 * N, dout[0], dout[1], dout[2], dout[3], dout[4], dout[5],
                    dst, c->stream);
    HCUDA(cudaGetLastError());
    for (int k = 0; k < 6; k++)
        if (outs[k])
            HCUDA(cudaMemcpyAsync(outs[k], dout[k], sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
    std::vector<int> own;
    int* hst = status;
    if (!hst) {
        own.resize(N);
        hst = own.data();
    }
    HCUDA(cudaMemcpyAsync(hst, dst, sizeof(int) * N, cudaMemcpyDeviceToHost, c->stream));
    HCUDA(cudaStreamSynchronize(c->stream));
    const int rc = first_error(hst, n);
    if (rc) c->err = "some points outside the table or with cv < 0 / cs^2 < 0 (see status)";
    return rc;
}

int helm_invert_T_batch(helm_ctx* c, long long n, const double* rho, const double* target, const double* abar,
                        const double* zbar, int from_entropy, double* T, double* p, double* e, double* cs,
                        double* cv, double* s, int* iters, int* status) {
    if (!c || n < 0 || (n > 0 && (!rho || !target || !abar || !zbar || !T))) return AMR_ERR_ARG;
    if (n == 0) return AMR_OK;
    const size_t N = (size_t)n;
    // 5 inputs (incl. T), 5 outputs, iterations and statuses (ints)
    const size_t ints_d = (2 * N * sizeof(int) + sizeof(double) - 1) / sizeof(double);
    if (int rc = ensure_stage(c, 10 * N + ints_d)) return rc;
    double* D = c->d_stage;
    const double* ins[5] = {rho, target, abar, zbar, T};
    for (int k = 0; k < 5; k++)
        HCUDA(cudaMemcpyAsync(D + k * N, ins[k], sizeof(double) * N, cudaMemcpyHostToDevice, c->stream));
    double* outs[5] = {p, e, cs, cv, s};
    double* dout[5];
    for (int k = 0; k < 5; k++) dout[k] = outs[k] ? D + (5 + k) * N : nullptr;
    int* dit = reinterpret_cast<int*>(D + 10 * N);
    int* dst = dit + N;
    launch_helm_invert(c->tab, n, D, D + N, D + 2 * N, D + 3 * N, from_entropy ? 1 : 0, D + 4 * N, dout[0], dout[1],
                       dout[2], dout[3], dout[4], dit, dst, c->stream);
    HCUDA(cudaGetLastError());
    HCUDA(cudaMemcpyAsync(T, D + 4 * N, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
    for (int k = 0; k < 5; k++)
        if (outs[k])
            HCUDA(cudaMemcpyAsync(outs[k], dout[k], sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
    if (iters) HCUDA(cudaMemcpyAsync(iters, dit, sizeof(int) * N, cudaMemcpyDeviceToHost, c->stream));
    std::vector<int> own;
    int* hst = status;
    if (!hst) {
        own.resize(N);
        hst = own.data();
    }
    HCUDA(cudaMemcpyAsync(hst, dst, sizeof(int) * N, cudaMemcpyDeviceToHost, c->stream));
    HCUDA(cudaStreamSynchronize(c->stream));
    const int rc = first_error(hst, n);
    if (rc) c->err = "some points failed the temperature inversion (see status)";
    return rc;
}

int helm_ztwd_batch(helm_ctx* c, long long n, const double* zbar, const double* rho, double* p, double* e) {
    if (!c || n < 0 || (n > 0 && (!zbar || !rho || !p || !e))) return AMR_ERR_ARG;
    if (n == 0) return AMR_OK;
    const size_t N = (size_t)n;
    if (int rc = ensure_stage(c, 4 * N)) return rc;
    double* D = c->d_stage;
    HCUDA(cudaMemcpyAsync(D, zbar, sizeof(double) * N, cudaMemcpyHostToDevice, c->stream));
    HCUDA(cudaMemcpyAsync(D + N, rho, sizeof(double) * N, cudaMemcpyHostToDevice, c->stream));
    launch_helm_ztwd(n, D, D + N, D + 2 * N, D + 3 * N, c->stream);
    HCUDA(cudaGetLastError());
    HCUDA(cudaMemcpyAsync(p, D + 2 * N, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
    HCUDA(cudaMemcpyAsync(e, D + 3 * N, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
    HCUDA(cudaStreamSynchronize(c->stream));
    return AMR_OK;
}

}  // extern "C"

namespace amr {
const HelmTable* helm_table_of(const helm_ctx* c) { return c ? &c->tab : nullptr; }
}  // namespace amr
