// Raw dumps of a reference octree (test infrastructure, shared by the
// oracle harnesses): every node's header, its GNX^3 state and, for Poisson
// nodes, its eight PNX^3 arrays, in depth-first pre-order; read by
// oracle/dumpio.py.  Include after the reference headers (GridNode,
// Poisson) with access control relaxed.
#pragma once

#include <stdio.h>
#include <stdlib.h>
#include <vector>

static void dump_node(FILE* fp, const GridNode* g, const Poisson* p) {
    int hdr[10];
    hdr[0] = g->get_level();
    for (int d = 0; d < 3; d++) hdr[1 + d] = g->get_location()[d];
    for (int d = 0; d < 3; d++) hdr[4 + d] = g->get_offset()[d];
    hdr[7] = g->age;
    int cm = 0, rm = 0;
    for (int c = 0; c < 8; c++) {
        if (g->get_child(c) != NULL) cm |= 1 << c;
        if (g->refine[c]) rm |= 1 << c;
    }
    hdr[8] = cm;
    hdr[9] = rm;
    fwrite(hdr, sizeof(int), 10, fp);
    const double h = g->get_dx();
    fwrite(&h, sizeof(double), 1, fp);
    std::vector<double> buf((size_t)STATE_NF * GNX * GNX * GNX);
    size_t n = 0;
    for (int f = 0; f < STATE_NF; f++)
        for (int k = 0; k < GNX; k++)
            for (int j = 0; j < GNX; j++)
                for (int i = 0; i < GNX; i++) buf[n++] = (*g)(i, j, k)[f];
    fwrite(buf.data(), sizeof(double), n, fp);
    if (p) {
        const Array3d<PReal, PNX, PNX, PNX>* arrs[8] = {&p->phi, &p->phi0, &p->dphi, &p->dphi1,
                                                         &p->S,   &p->fx,   &p->fy,   &p->fz};
        std::vector<double> pb((size_t)PNX * PNX * PNX);
        for (int a = 0; a < 8; a++) {
            size_t m = 0;
            for (int k = 0; k < PNX; k++)
                for (int j = 0; j < PNX; j++)
                    for (int i = 0; i < PNX; i++) pb[m++] = (*arrs[a])(i, j, k);
            fwrite(pb.data(), sizeof(double), m, fp);
        }
    }
    for (int c = 0; c < 8; c++) {
        const GridNode* ch = static_cast<const GridNode*>(g->get_child(c));
        if (ch) dump_node(fp, ch, p ? static_cast<const Poisson*>(g->get_child(c)) : NULL);
    }
}

// file layout: "AMRDUMP1", int32[8] {bw, gnx, nf, pnx, has_poisson, nnodes,
// nrecords_extra, reserved}, double time, then node records, then the root
// flow-off vector FO[nf], then an extra double array (per-step dt, errors ...).
static void dump(const char* path, const GridNode* root, const Poisson* proot, double time,
                 const std::vector<double>& extra) {
    FILE* fp = fopen(path, "wb");
    if (!fp) {
        perror(path);
        exit(3);
    }
    fwrite("AMRDUMP1", 1, 8, fp);
    int hdr[8] = {BW, GNX, STATE_NF, PNX, proot != NULL, root->get_node_cnt(), (int)extra.size(), 0};
    fwrite(hdr, sizeof(int), 8, fp);
    fwrite(&time, sizeof(double), 1, fp);
    dump_node(fp, root, proot);
    const State fo = root->flow_off();
    for (int f = 0; f < STATE_NF; f++) {
        const double v = fo[f];
        fwrite(&v, sizeof(double), 1, fp);
    }
    if (!extra.empty()) fwrite(extra.data(), sizeof(double), extra.size(), fp);
    fclose(fp);
}

