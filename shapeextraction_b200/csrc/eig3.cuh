// 3x3 symmetric eigensolver shared by the exact search kernel and the
// reference-compatible search kernel.
#pragma once
#include <cuda_runtime.h>

namespace shapex {

// ---- 3x3 symmetric eigensolver: cyclic Jacobi (Golub & Van Loan, Matrix
// Computations, 4th ed., Alg. 8.5.2 sym.schur2 + 8.5.3), explicit indices ----
template <typename T>
__device__ __forceinline__ T rsqrt_t(T x);
template <>
__device__ __forceinline__ float rsqrt_t<float>(float x) { return 1.0f / sqrtf(x); }
template <>
__device__ __forceinline__ double rsqrt_t<double>(double x) { return 1.0 / sqrt(x); }

template <int P, int Q, typename T>
__device__ __forceinline__ void jrot(T (&A)[3][3], T (&V)[3][3]) {
    const T apq = A[P][Q];
    if (apq == T(0)) return;
    constexpr int R = 3 - P - Q;
    const T theta = (A[Q][Q] - A[P][P]) / (T(2) * apq);
    const T at = fabs(theta);
    T t;
    if (at > T(1e15)) t = T(0.5) / theta;
    else t = (theta >= T(0) ? T(1) : T(-1)) / (at + sqrt(theta * theta + T(1)));
    const T c = rsqrt_t<T>(t * t + T(1));
    const T s = t * c;
    A[P][P] -= t * apq;
    A[Q][Q] += t * apq;
    A[P][Q] = A[Q][P] = T(0);
    const T arp = A[R][P], arq = A[R][Q];
    A[R][P] = A[P][R] = c * arp - s * arq;
    A[R][Q] = A[Q][R] = s * arp + c * arq;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const T vkp = V[k][P], vkq = V[k][Q];
        V[k][P] = c * vkp - s * vkq;
        V[k][Q] = s * vkp + c * vkq;
    }
}

// Returns the eigenvector of the smallest eigenvalue in n, and the ascending
// eigenvalues in w.
template <typename T>
__device__ __forceinline__ void eig3(const T (&C)[6], T (&w)[3], T (&n)[3]) {
    T A[3][3] = {{C[0], C[1], C[2]}, {C[1], C[3], C[4]}, {C[2], C[4], C[5]}};
    T V[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    const T eps2 = sizeof(T) == 4 ? T(1e-14) : T(1e-30);
    const int sweeps = sizeof(T) == 4 ? 12 : 20;
    for (int s = 0; s < sweeps; ++s) {
        const T off = A[0][1] * A[0][1] + A[0][2] * A[0][2] + A[1][2] * A[1][2];
        const T dia = A[0][0] * A[0][0] + A[1][1] * A[1][1] + A[2][2] * A[2][2];
        if (!(off > eps2 * dia)) break;
        jrot<0, 1>(A, V);
        jrot<0, 2>(A, V);
        jrot<1, 2>(A, V);
    }
    const T e0 = A[0][0], e1 = A[1][1], e2 = A[2][2];
    // ascending order with a stable tie rule (lower column first)
    int i0 = 0, i1 = 1, i2 = 2;
    T a0 = e0, a1 = e1, a2 = e2;
    if (a1 < a0) { T t = a0; a0 = a1; a1 = t; int ti = i0; i0 = i1; i1 = ti; }
    if (a2 < a1) { T t = a1; a1 = a2; a2 = t; int ti = i1; i1 = i2; i2 = ti; }
    if (a1 < a0) { T t = a0; a0 = a1; a1 = t; int ti = i0; i0 = i1; i1 = ti; }
    w[0] = a0; w[1] = a1; w[2] = a2;
    n[0] = i0 == 0 ? V[0][0] : (i0 == 1 ? V[0][1] : V[0][2]);
    n[1] = i0 == 0 ? V[1][0] : (i0 == 1 ? V[1][1] : V[1][2]);
    n[2] = i0 == 0 ? V[2][0] : (i0 == 1 ? V[2][1] : V[2][2]);
}

}  // namespace shapex
