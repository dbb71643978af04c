// Checkpoint files in the reference's binary format (X.*.chk):
// Binary::write / Binary::read (binary/binary.cpp:70-94, 175-203, the root
// header of the BINARY build), GridNode::write / read
// (grid/grid_node.cpp:29-57) and Grid::write / read (grid/grid.cpp:104-146).
//
// File: [Binary header: bool, 15 doubles (l1x, h, M1, fill_factor, n, R1,
// q, a, K1, K2, phi0_1, phi0_2, Omega, phase, Omega0), 2 ints (accretor and
// donor type)], then the nodes in depth-first pre-order, each
//   double h, h0, time; 3 x (int offset, double origin); double FO[NF];
//   double U[i][j][k][l] (GNX^3 x NF, i outermost, field innermost);
//   bool child[8]; double refine_alpha; int age
// written field by field with no padding (fwrite of each member).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "context.h"

using namespace amr;

#define TRY(x)                        \
    do {                              \
        int rc_ = (x);                \
        if (rc_ != AMR_OK) return rc_; \
    } while (0)

namespace {

struct File {
    FILE* fp = nullptr;
    ~File() {
        if (fp) fclose(fp);
    }
};

template <typename T>
bool put(FILE* fp, const T& v) {
    return fwrite(&v, sizeof(T), 1, fp) == 1;
}
template <typename T>
bool get(FILE* fp, T* v) {
    return fread(v, sizeof(T), 1, fp) == 1;
}

bool put_header(FILE* fp, const amr_binary_header* h) {
    const unsigned char dummy = h->dummy;  // written as read (uninitialised in the reference)
    bool ok = fwrite(&dummy, 1, 1, fp) == 1;
    const double d[15] = {h->l1x, h->h,    h->M1,     h->fill_factor, h->n,     h->R1,    h->q,     h->a,
                          h->K1,  h->K2,   h->phi0_1, h->phi0_2,      h->Omega, h->phase, h->Omega0};
    for (double x : d) ok = ok && put(fp, x);
    ok = ok && put(fp, h->accretor_type) && put(fp, h->donor_type);
    return ok;
}

bool get_header(FILE* fp, amr_binary_header* h) {
    unsigned char dummy = 0;
    bool ok = fread(&dummy, 1, 1, fp) == 1;
    double d[15];
    for (double& x : d) ok = ok && get(fp, &x);
    int at = 0, dt = 0;
    ok = ok && get(fp, &at) && get(fp, &dt);
    if (!ok) return false;
    h->dummy = dummy;
    h->l1x = d[0], h->h = d[1], h->M1 = d[2], h->fill_factor = d[3], h->n = d[4], h->R1 = d[5], h->q = d[6];
    h->a = d[7], h->K1 = d[8], h->K2 = d[9], h->phi0_1 = d[10], h->phi0_2 = d[11], h->Omega = d[12];
    h->phase = d[13], h->Omega0 = d[14];
    h->accretor_type = at, h->donor_type = dt;
    return true;
}

struct NodeRec {
    int level, loc[3], age;
    int offset[3];
    double h, time;
    double fo[32];
    std::vector<double> U;  // [nf][gnx^3], our layout
};

// one node record and its subtree, depth first
int read_node(amr_ctx* c, FILE* fp, int level, const int* loc, const int* exp_off, std::vector<NodeRec>& out) {
    const Geom& g = c->geom;
    NodeRec r;
    r.level = level;
    for (int d = 0; d < 3; d++) r.loc[d] = loc[d];
    double h0;
    bool ok = get(fp, &r.h) && get(fp, &h0) && get(fp, &r.time);
    for (int d = 0; d < 3 && ok; d++) {
        double origin;
        ok = get(fp, &r.offset[d]) && get(fp, &origin);
    }
    for (int l = 0; l < g.nf && ok; l++) ok = get(fp, &r.fo[l]);
    if (!ok) {
        c->err = "checkpoint: truncated node header";
        return AMR_ERR_STATE;
    }
    for (int d = 0; d < 3; d++)
        if (r.offset[d] != exp_off[d]) {
            c->err = "checkpoint: brick offsets do not match this configuration (BW, GNX)";
            return AMR_ERR_STATE;
        }
    const int gnx = g.gnx, nf = g.nf;
    std::vector<double> cells((size_t)g.gnx3 * nf);
    if (fread(cells.data(), sizeof(double), cells.size(), fp) != cells.size()) {
        c->err = "checkpoint: truncated cell data";
        return AMR_ERR_STATE;
    }
    r.U.resize(cells.size());
    size_t n = 0;
    for (int i = 0; i < gnx; i++)
        for (int j = 0; j < gnx; j++)
            for (int k = 0; k < gnx; k++)
                for (int l = 0; l < nf; l++) r.U[(size_t)l * g.gnx3 + (k * gnx + j) * gnx + i] = cells[n++];
    unsigned char child[8];
    double alpha;
    if (fread(child, 1, 8, fp) != 8 || !get(fp, &alpha) || !get(fp, &r.age)) {
        c->err = "checkpoint: truncated node trailer";
        return AMR_ERR_STATE;
    }
    c->chk_refine_alpha = alpha;  // GridNode::refine_alpha is one static: every node writes the same
    out.push_back(std::move(r));
    for (int q = 0; q < 8; q++) {
        if (!child[q]) continue;
        const int cl[3] = {2 * loc[0] + (q & 1), 2 * loc[1] + ((q >> 1) & 1), 2 * loc[2] + ((q >> 2) & 1)};
        // GridNode::create_child (grid_node.cpp:276): 2 offset + BW + c (GNX - 2 BW)
        const int co[3] = {2 * exp_off[0] + g.bw + (q & 1) * g.nx, 2 * exp_off[1] + g.bw + ((q >> 1) & 1) * g.nx,
                           2 * exp_off[2] + g.bw + ((q >> 2) & 1) * g.nx};
        TRY(read_node(c, fp, level + 1, cl, co, out));
    }
    return AMR_OK;
}

}  // namespace

extern "C" {

int amr_write_checkpoint(amr_ctx* c, const char* path, const amr_binary_header* hdr, double refine_alpha) {
    if (!c || !path) return AMR_ERR_ARG;
    if (!c->has_device) {
        c->err = "context has no device pool";
        return AMR_ERR_NODEVICE;
    }
    const Geom& g = c->geom;
    const int n = (int)c->order.size();
    std::vector<double> U((size_t)n * g.ucount);
    TRY(amr_download_state(c, U.data()));
    double fo[64];
    TRY(amr_get_flow_off(c, fo));
    File f;
    f.fp = fopen(path, "wb");
    if (!f.fp) {
        c->err = std::string("cannot open ") + path;
        return AMR_ERR_ARG;
    }
    if (refine_alpha < 0.0) refine_alpha = c->chk_refine_alpha;
    bool ok = !hdr || put_header(f.fp, hdr);
    std::vector<double> cells((size_t)g.gnx3 * g.nf);
    for (int e = 0; e < n && ok; e++) {
        const Node* nd = c->order[e];
        ok = put(f.fp, nd->h) && put(f.fp, g.h0) && put(f.fp, c->time);
        for (int d = 0; d < 3 && ok; d++) ok = put(f.fp, nd->off[d]) && put(f.fp, g.origin[d]);
        for (int l = 0; l < g.nf && ok; l++) ok = put(f.fp, e == 0 ? fo[l] : 0.0);  // FO: root only
        const double* Ub = U.data() + (size_t)e * g.ucount;
        size_t m = 0;
        for (int i = 0; i < g.gnx; i++)
            for (int j = 0; j < g.gnx; j++)
                for (int k = 0; k < g.gnx; k++)
                    for (int l = 0; l < g.nf; l++) cells[m++] = Ub[(size_t)l * g.gnx3 + (k * g.gnx + j) * g.gnx + i];
        ok = ok && fwrite(cells.data(), sizeof(double), cells.size(), f.fp) == cells.size();
        unsigned char child[8];
        for (int q = 0; q < 8; q++) child[q] = nd->child[q] ? 1 : 0;
        ok = ok && fwrite(child, 1, 8, f.fp) == 8 && put(f.fp, refine_alpha) && put(f.fp, nd->age);
    }
    if (!ok) {
        c->err = std::string("write failed: ") + path;
        return AMR_ERR_STATE;
    }
    return AMR_OK;
}

int amr_read_checkpoint(amr_ctx* c, const char* path, amr_binary_header* hdr) {
    if (!c || !path) return AMR_ERR_ARG;
    if (!c->has_device) {
        c->err = "context has no device pool";
        return AMR_ERR_NODEVICE;
    }
    File f;
    f.fp = fopen(path, "rb");
    if (!f.fp) {
        c->err = std::string("cannot open ") + path;
        return AMR_ERR_ARG;
    }
    if (hdr && !get_header(f.fp, hdr)) {
        c->err = "checkpoint: truncated Binary header";
        return AMR_ERR_STATE;
    }
    std::vector<NodeRec> recs;
    const int loc0[3] = {0, 0, 0}, off0[3] = {0, 0, 0};
    TRY(read_node(c, f.fp, 0, loc0, off0, recs));
    if (fgetc(f.fp) != EOF) {
        c->err = "checkpoint: trailing bytes (NF, GNX or the Binary header do not match this configuration)";
        return AMR_ERR_STATE;
    }
    const int n = (int)recs.size();
    std::vector<int> level(n), loc(3 * (size_t)n), age(n);
    for (int e = 0; e < n; e++) {
        level[e] = recs[e].level;
        for (int d = 0; d < 3; d++) loc[3 * e + d] = recs[e].loc[d];
        age[e] = recs[e].age;
    }
    TRY(amr_load_tree(c, n, level.data(), loc.data(), age.data()));
    const Geom& g = c->geom;
    std::vector<double> U((size_t)n * g.ucount);
    for (int e = 0; e < n; e++) std::memcpy(U.data() + (size_t)e * g.ucount, recs[e].U.data(), sizeof(double) * g.ucount);
    TRY(amr_upload_state(c, U.data()));
    double fo[64] = {0};
    for (int l = 0; l < g.nf; l++) fo[l] = recs[0].fo[l];
    TRY(amr_set_flow_off(c, fo));
    return amr_set_time(c, recs[0].time);
}

// Headless output (the per-brick data GridNode::output writes to Silo,
// grid/grid_node.cpp:1422-1487, without the Silo library): "AMRB200O",
// int32 {nf, nx, bw, nbricks, has_phi, 0, 0, 0}, double time, then per brick
// in depth-first pre-order int32 {level, loc[3], offset[3], age,
// child_mask}, double h, the interior state [nf][nx][nx][nx] and, with
// self-gravity, the interior potential [nx][nx][nx].
int amr_write_output(amr_ctx* c, const char* path) {
    if (!c || !path) return AMR_ERR_ARG;
    if (!c->has_device) {
        c->err = "context has no device pool";
        return AMR_ERR_NODEVICE;
    }
    const Geom& g = c->geom;
    const int n = (int)c->order.size();
    std::vector<double> U((size_t)n * g.ucount);
    TRY(amr_download_state(c, U.data()));
    const bool phi = has_gravity(c) && c->d_bphi != nullptr;
    std::vector<double> P;
    if (phi) {
        P.resize((size_t)8 * n * g.pnx3);
        TRY(amr_download_poisson(c, P.data()));
    }
    File f;
    f.fp = fopen(path, "wb");
    if (!f.fp) {
        c->err = std::string("cannot open ") + path;
        return AMR_ERR_ARG;
    }
    const int hdr[8] = {g.nf, g.nx, g.bw, n, phi ? 1 : 0, 0, 0, 0};
    bool ok = fwrite("AMRB200O", 1, 8, f.fp) == 8 && fwrite(hdr, sizeof(int), 8, f.fp) == 8 && put(f.fp, c->time);
    std::vector<double> buf((size_t)g.nf * g.nx * g.nx * g.nx);
    for (int e = 0; e < n && ok; e++) {
        const Node* nd = c->order[e];
        int cm = 0;
        for (int q = 0; q < 8; q++) cm |= nd->child[q] ? 1 << q : 0;
        const int rec[9] = {nd->level, nd->loc[0], nd->loc[1], nd->loc[2], nd->off[0], nd->off[1], nd->off[2],
                            nd->age, cm};
        ok = fwrite(rec, sizeof(int), 9, f.fp) == 9 && put(f.fp, nd->h);
        const double* Ub = U.data() + (size_t)e * g.ucount;
        size_t m = 0;
        for (int l = 0; l < g.nf; l++)
            for (int k = g.bw; k < g.bw + g.nx; k++)
                for (int j = g.bw; j < g.bw + g.nx; j++)
                    for (int i = g.bw; i < g.bw + g.nx; i++) buf[m++] = Ub[(size_t)l * g.gnx3 + (k * g.gnx + j) * g.gnx + i];
        ok = ok && fwrite(buf.data(), sizeof(double), m, f.fp) == m;
        if (phi && ok) {
            const double* pb = P.data() + (size_t)e * g.pnx3;  // phi is the first of the 8 arrays
            m = 0;
            for (int k = 1; k <= g.nx; k++)
                for (int j = 1; j <= g.nx; j++)
                    for (int i = 1; i <= g.nx; i++) buf[m++] = pb[(k * g.pnx + j) * g.pnx + i];
            ok = fwrite(buf.data(), sizeof(double), m, f.fp) == m;
        }
    }
    if (!ok) {
        c->err = std::string("write failed: ") + path;
        return AMR_ERR_STATE;
    }
    return AMR_OK;
}

}  // extern "C"
