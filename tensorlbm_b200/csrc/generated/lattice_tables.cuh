// Generated by tensorlbm_b200/csrc/gen_tables.py - do not edit.
#pragma once

struct D2Q9 {
  static constexpr int Q = 9;
  static constexpr int DIM = 2;
  __host__ __device__ static constexpr int cx(int q) { constexpr int t[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1}; return t[q]; }
  __host__ __device__ static constexpr int cy(int q) { constexpr int t[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1}; return t[q]; }
  __host__ __device__ static constexpr int cz(int q) { constexpr int t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}; return t[q]; }
  __host__ __device__ static constexpr int opp(int q) { constexpr int t[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6}; return t[q]; }
  __host__ __device__ static constexpr double w(int q) { constexpr double t[9] = {0.4444444444444444, 0.1111111111111111, 0.1111111111111111, 0.1111111111111111, 0.1111111111111111, 0.027777777777777776, 0.027777777777777776, 0.027777777777777776, 0.027777777777777776}; return t[q]; }
};

struct D3Q19 {
  static constexpr int Q = 19;
  static constexpr int DIM = 3;
  __host__ __device__ static constexpr int cx(int q) { constexpr int t[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0}; return t[q]; }
  __host__ __device__ static constexpr int cy(int q) { constexpr int t[19] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1}; return t[q]; }
  __host__ __device__ static constexpr int cz(int q) { constexpr int t[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1}; return t[q]; }
  __host__ __device__ static constexpr int opp(int q) { constexpr int t[19] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17}; return t[q]; }
  __host__ __device__ static constexpr double w(int q) { constexpr double t[19] = {0.3333333333333333, 0.05555555555555555, 0.05555555555555555, 0.05555555555555555, 0.05555555555555555, 0.05555555555555555, 0.05555555555555555, 0.027777777777777776, 0.027777777777777776, 0.027777777777777776, 0.027777777777777776, 0.027777777777777776, 0.027777777777777776, 0.027777777777777776, 0.027777777777777776, 0.027777777777777776, 0.027777777777777776, 0.027777777777777776, 0.027777777777777776}; return t[q]; }
};

struct D3Q27 {
  static constexpr int Q = 27;
  static constexpr int DIM = 3;
  __host__ __device__ static constexpr int cx(int q) { constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1}; return t[q]; }
  __host__ __device__ static constexpr int cy(int q) { constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, 1, -1, -1, 1, 1, -1, -1}; return t[q]; }
  __host__ __device__ static constexpr int cz(int q) { constexpr int t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, 1, 1, -1, -1, -1, -1}; return t[q]; }
  __host__ __device__ static constexpr int opp(int q) { constexpr int t[27] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15, 26, 25, 24, 23, 22, 21, 20, 19}; return t[q]; }
  __host__ __device__ static constexpr double w(int q) { constexpr double t[27] = {0.2962962962962963, 0.07407407407407407, 0.07407407407407407, 0.07407407407407407, 0.07407407407407407, 0.07407407407407407, 0.07407407407407407, 0.018518518518518517, 0.018518518518518517, 0.018518518518518517, 0.018518518518518517, 0.018518518518518517, 0.018518518518518517, 0.018518518518518517, 0.018518518518518517, 0.018518518518518517, 0.018518518518518517, 0.018518518518518517, 0.018518518518518517, 0.004629629629629629, 0.004629629629629629, 0.004629629629629629, 0.004629629629629629, 0.004629629629629629, 0.004629629629629629, 0.004629629629629629, 0.004629629629629629}; return t[q]; }
};
