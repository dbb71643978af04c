// Face reconstruction along one pencil, streamed cell by cell: the left and
// right primitive states of faces bw .. gnx-bw, in the order the flux loop
// of Grid::compute_{x,y,z}_flux (grid.cpp:215-302) and Grid::max_dt
// (grid.cpp:422-483) visits them.  Two methods, as Reconstruct::operator()
// (reconstruct.cpp:92-102) selects them:
//
//   RECON_MINMOD  Reconstruct::minmod (reconstruct.cpp:60-71):
//                 s = minmod_theta(q[i+1]-q[i], q[i]-q[i-1], theta);
//                 ql[f] = q[f-1] + s[f-1]/2, qr[f] = q[f] - s[f]/2.
//   RECON_PPM     Reconstruct::ppm (reconstruct.cpp:22-58) as called,
//                 ppm(q0, qr, ql) (reconstruct.cpp:94): slopes minmod_theta
//                 with theta 2; interface I[i] = (q[i]+q[i+1])/2 +
//                 (s[i]-s[i+1])/6 to the right of cell i; each cell's edges
//                 (I[i-1], I[i]) monotonised (Colella-Woodward); face f gets
//                 the right edge of cell f-1 and the left edge of cell f (the
//                 final shift of reconstruct.cpp:55-57).  Needs bw >= 3.  The
//                 Euler state has no low-order or smooth field
//                 (euler/state.h:37-42), so all fields take both steps.
//
// The caller supplies load(n, q): the primitives of cell n of the pencil.
// Arithmetic keeps the reference's operation order (FP64 instantiations are
// compiled without FMA contraction).
#pragma once

#include "euler_state.cuh"

namespace amr {

constexpr int RECON_MINMOD = 0;
constexpr int RECON_PPM = 1;

template <typename T, int R>
struct PencilRecon;

template <typename T>
struct PencilRecon<T, RECON_MINMOD> {
    T w1[NF_EULER], w2[NF_EULER], w3[NF_EULER];  // cells f-2, f-1, f (before next())
    T sR[NF_EULER];                              // slope of cell f-1
    T th;

    // ready for face bw: cells bw-2 .. bw in the window, slope of cell bw-1
    template <class Load>
    __device__ __forceinline__ void begin(Load& load, int bw, T theta) {
        th = theta;
        load(bw - 2, w1);
        load(bw - 1, w2);
        load(bw, w3);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) sR[l] = minmod_theta(w3[l] - w2[l], w2[l] - w1[l], th);
    }
    // states of face f (called for f = bw, bw+1, ...): ql from cell f-1, qr from cell f
    template <class Load>
    __device__ __forceinline__ void next(Load& load, int f, T* ql, T* qr) {
        T w4[NF_EULER];
        load(f + 1, w4);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) {
            const T sL = sR[l];                                     // s[f-1]
            sR[l] = minmod_theta(w4[l] - w3[l], w3[l] - w2[l], th);  // s[f]
            ql[l] = w2[l] + sL / T(2);
            qr[l] = w3[l] - sR[l] / T(2);
            w1[l] = w2[l];
            w2[l] = w3[l];
            w3[l] = w4[l];
        }
    }
};

template <typename T>
struct PencilRecon<T, RECON_PPM> {
    T qc[NF_EULER], qn[NF_EULER];  // cells c, c+1
    T sc[NF_EULER];                // slope of cell c
    T Ip[NF_EULER];                // interface to the right of cell c-1
    T Rm[NF_EULER];                // monotonised right edge of cell c-1
    int c;                         // next cell to monotonise

    // Cell c: load c+2, slope of c+1, interface right of c, monotonise c.
    // Lm gets the left edge of cell c; Rm becomes its right edge.
    template <class Load>
    __device__ __forceinline__ void advance(Load& load, T* Lm) {
        T q2[NF_EULER];
        load(c + 2, q2);
        const T six = T(1.0 / 6.0);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) {
            const T sn = minmod_theta(q2[l] - qn[l], qn[l] - qc[l], T(2.0));
            T Ic = (qc[l] + qn[l]) * T(0.5);
            Ic += (sc[l] - sn) * six;
            // reconstruct.cpp:40-53, ql = Ip, qr = Ic, q0 = qc
            T lo = Ip[l], hi = Ic;
            const T q0 = qc[l];
            const T tmp1 = hi - lo;
            const T tmp2 = hi + lo;
            if ((hi - q0) * (q0 - lo) <= T(0)) {
                hi = lo = q0;
            } else if (tmp1 * (q0 - T(0.5) * tmp2) > six * tmp1 * tmp1) {
                lo = T(3.0) * q0 - T(2.0) * hi;
            } else if (-six * tmp1 * tmp1 > tmp1 * (q0 - T(0.5) * tmp2)) {
                hi = T(3.0) * q0 - T(2.0) * lo;
            }
            Lm[l] = lo;
            Rm[l] = hi;
            Ip[l] = Ic;
            sc[l] = sn;
            qc[l] = qn[l];
            qn[l] = q2[l];
        }
        c++;
    }

    template <class Load>
    __device__ __forceinline__ void begin(Load& load, int bw, T) {
        T q0[NF_EULER], q1[NF_EULER];
        load(0, q0);
        load(1, q1);
        load(2, qc);
        load(3, qn);
        const T six = T(1.0 / 6.0);
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) {
            const T s1 = minmod_theta(qc[l] - q1[l], q1[l] - q0[l], T(2.0));
            sc[l] = minmod_theta(qn[l] - qc[l], qc[l] - q1[l], T(2.0));
            T I1 = (q1[l] + qc[l]) * T(0.5);
            I1 += (s1 - sc[l]) * six;
            Ip[l] = I1;
        }
        c = 2;
        T Lm[NF_EULER];
        while (c < bw) advance(load, Lm);  // leaves Rm = right edge of cell bw-1
    }

    template <class Load>
    __device__ __forceinline__ void next(Load& load, int, T* ql, T* qr) {
#pragma unroll
        for (int l = 0; l < NF_EULER; l++) ql[l] = Rm[l];  // right edge of cell f-1
        advance(load, qr);                                  // left edge of cell f
    }
};

}  // namespace amr
