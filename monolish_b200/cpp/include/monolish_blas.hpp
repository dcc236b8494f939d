// monolish-compatible BLAS for the sparse solve path (device-resident
// operands; every call runs an sm_100a kernel through include/mlsh.h).
//
//   matvec  include/monolish/blas/monolish_matvec_blas.hpp:3972 (CRS x vector),
//           alpha/beta overload src/blas/matrix/matvec/matvec_blas.cpp:3853
//   matvec_T (CRS^T x vector)
//   dot, nrm2, axpy, xpay, axpyz, copy
//           include/monolish/blas/monolish_vector_blas.hpp
#pragma once
#include "monolish/common/monolish_common.hpp"

namespace monolish {
namespace blas {

void matvec(const matrix::CRS<double> &A, const vector<double> &x, vector<double> &y);
void matvec(const matrix::CRS<float> &A, const vector<float> &x, vector<float> &y);
void matvec(const double &a, const matrix::CRS<double> &A, const vector<double> &x,
            const double &b, vector<double> &y);
void matvec(const float &a, const matrix::CRS<float> &A, const vector<float> &x,
            const float &b, vector<float> &y);

// y = A^T x  (include/monolish/blas/monolish_matvec_blas.hpp:4283,
// src/blas/matrix/matvec/crs_matvec.hpp:88-98)
void matvec_T(const matrix::CRS<double> &A, const vector<double> &x, vector<double> &y);
void matvec_T(const matrix::CRS<float> &A, const vector<float> &x, vector<float> &y);

double dot(const vector<double> &x, const vector<double> &y);
float dot(const vector<float> &x, const vector<float> &y);
void dot(const vector<double> &x, const vector<double> &y, double &ans);
void dot(const vector<float> &x, const vector<float> &y, float &ans);

double nrm2(const vector<double> &x);
float nrm2(const vector<float> &x);
void nrm2(const vector<double> &x, double &ans);
void nrm2(const vector<float> &x, float &ans);

void axpy(const double alpha, const vector<double> &x, vector<double> &y);
void axpy(const float alpha, const vector<float> &x, vector<float> &y);
void xpay(const double alpha, const vector<double> &x, vector<double> &y);
void xpay(const float alpha, const vector<float> &x, vector<float> &y);
void axpyz(const double alpha, const vector<double> &x, const vector<double> &y,
           vector<double> &z);
void axpyz(const float alpha, const vector<float> &x, const vector<float> &y,
           vector<float> &z);
void copy(const vector<double> &x, vector<double> &y);
void copy(const vector<float> &x, vector<float> &y);

}  // namespace blas
}  // namespace monolish
