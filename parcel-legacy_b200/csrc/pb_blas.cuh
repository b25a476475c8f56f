// pb_blas.cuh -- host launchers of the vector kernels (pb_blas.cu).
#pragma once

#include "pb_device.cuh"

namespace pb {

// A scalar coefficient: either an immediate value or mul * (*p) read on the device.
struct Coef {
  const double* p = nullptr;
  double v = 0.0;
  double mul = 1.0;
};
inline Coef cimm(double v) { Coef c; c.v = v; return c; }
inline Coef cdev(const double* p, double mul = 1.0) { Coef c; c.p = p; c.mul = mul; return c; }

// Which operands a fused dot multiplies: 0 = out, 1 = x0, 2 = x1, 3 = x2, 4 = d0, 5 = d1.
struct DotSel {
  int a[3] = {0, 0, 0};
  int b[3] = {0, 0, 0};
};

template <class T>
void lincomb(int64_t n, T* out, const T* x0, Coef c0, const T* x1, Coef c1, const T* x2, Coef c2,
             const int* gate, cudaStream_t st);
template <class T>
void lincomb_dot(int64_t n, T* out, const T* x0, Coef c0, const T* x1, Coef c1, const T* x2,
                 Coef c2, const T* d0, const T* d1, DotSel sel, int nd, const Red& red,
                 const int* gate, cudaStream_t st);
template <class T>
void cg_axpy2(int64_t n, T* x, T* p, const T* s, const KState* st, const int* gate, cudaStream_t s_);
template <class T>
void scale(int64_t n, T* s, const T* d, const T* r, const int* gate, cudaStream_t st);
template <class T>
void multidot(int64_t n, int j, const T* w, const T* V, int64_t ldv, const Red& red, const int* gate,
              cudaStream_t st);
template <class T>
void cgs_update(int64_t n, int j, T* w, const T* V, int64_t ldv, const double* hcol, const Red& red,
                const int* gate, cudaStream_t st);
template <class T>
void sum_vec(int64_t n, T* v0, const T* V, int64_t ldv, const double* y, const KState* st,
             const int* gate, cudaStream_t s_);
void gm_backsolve(const double* h, const double* e, double* y, int m0, KState* st, const int* gate,
                  cudaStream_t s_);
void gm_post(KState* st, int m, int itrmax, cudaStream_t s_);
void fill(int64_t n, double* p, double v, cudaStream_t st);
template <class TO, class TI>
void convert(int64_t n, TO* o, const TI* in, cudaStream_t st);
template <class T>
void scatter_perm(int n, T* outp, const double* in, const int* perm, cudaStream_t st);
template <class T>
void gather_perm(int n, double* out, const T* inp, const int* perm, cudaStream_t st);

}  // namespace pb
