// Test harness around the reference Helmholtz EOS (helmholtz/helmeos.cpp),
// compiled unpatched from the reference tree by oracle/build_ref.py.  Test
// infrastructure only.
//
// The reference reads helmholtz.table from the working directory in a
// static constructor (helmeos.cpp:73-130), so run this with the table there.
//
//   helm_harness fwd IN OUT [cm g s K]
//       IN:  int64 n, then n records of (rho, T, abar, zbar) doubles
//       OUT: n records of (p, e, cs, cv, s, dsdt) doubles   (helmholtz_eos)
//   helm_harness inv IN OUT [cm g s K]
//       IN:  int64 n, then n records of (rho, e, abar, zbar, T_guess) doubles
//       OUT: n records of (T, p, e, cs, cv, s) doubles       (helmholtz_compute_T)
//   helm_harness invs IN OUT [cm g s K]
//       the same with the entropy as target (helmholtz_compute_T(eos, true))
//
// The optional unit factors go to helmholtz_set_cgs_units first.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "helmholtz.h"

static std::vector<double> read_records(const char* path, int width, int64_t* n_out) {
    FILE* f = fopen(path, "rb");
    if (!f) {
        perror(path);
        exit(2);
    }
    int64_t n = 0;
    if (fread(&n, sizeof(n), 1, f) != 1) exit(2);
    std::vector<double> v((size_t)n * width);
    if (n && fread(v.data(), sizeof(double), v.size(), f) != v.size()) exit(2);
    fclose(f);
    *n_out = n;
    return v;
}

static void write_records(const char* path, const std::vector<double>& v) {
    FILE* f = fopen(path, "wb");
    if (!f) {
        perror(path);
        exit(2);
    }
    if (!v.empty()) fwrite(v.data(), sizeof(double), v.size(), f);
    fclose(f);
}

int main(int argc, char** argv) {
    if (argc != 4 && argc != 8) {
        fprintf(stderr, "usage: helm_harness fwd|inv IN OUT [cm g s K]\n");
        return 2;
    }
    if (argc == 8) helmholtz_set_cgs_units(atof(argv[4]), atof(argv[5]), atof(argv[6]), atof(argv[7]));
    int64_t n = 0;
    if (!strcmp(argv[1], "fwd")) {
        std::vector<double> in = read_records(argv[2], 4, &n), out((size_t)n * 6);
        for (int64_t q = 0; q < n; q++) {
            eos_t e;
            memset(&e, 0, sizeof(e));
            e.rho = in[4 * q + 0];
            e.T = in[4 * q + 1];
            e.abar = in[4 * q + 2];
            e.zbar = in[4 * q + 3];
            helmholtz_eos(&e);
            double* o = &out[6 * q];
            o[0] = e.p;
            o[1] = e.e;
            o[2] = e.cs;
            o[3] = e.cv;
            o[4] = e.s;
            o[5] = e.dsdt;
        }
        write_records(argv[3], out);
    } else if (!strcmp(argv[1], "inv") || !strcmp(argv[1], "invs")) {
        const bool from_entropy = !strcmp(argv[1], "invs");
        std::vector<double> in = read_records(argv[2], 5, &n), out((size_t)n * 6);
        for (int64_t q = 0; q < n; q++) {
            eos_t e;
            memset(&e, 0, sizeof(e));
            e.rho = in[5 * q + 0];
            if (from_entropy) {
                e.s = in[5 * q + 1];
            } else {
                e.e = in[5 * q + 1];
            }
            e.abar = in[5 * q + 2];
            e.zbar = in[5 * q + 3];
            e.T = in[5 * q + 4];
            helmholtz_compute_T(&e, from_entropy);
            double* o = &out[6 * q];
            o[0] = e.T;
            o[1] = e.p;
            o[2] = e.e;
            o[3] = e.cs;
            o[4] = e.cv;
            o[5] = e.s;
        }
        write_records(argv[3], out);
    } else {
        fprintf(stderr, "unknown mode %s\n", argv[1]);
        return 2;
    }
    return 0;
}
