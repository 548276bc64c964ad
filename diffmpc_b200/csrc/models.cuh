// Continuous-time dynamics and the one-step integrator, templated on the
// scalar type (double, Dual, HDual) so the same code gives values, Jacobian
// columns and mixed second derivatives.
//
//   linear      diffmpc/dynamics/linear_dynamics.py:46-70      x' = A x + B u + b
//   quadrotor   diffmpc/dynamics/quadrotor_dynamics.py:84-133  [p, v, q, w], [thrust, tau]
//   spacecraft  diffmpc/dynamics/spacecraft_dynamics.py:31-66  w' = J^-1 (tau - w x J w)
//   attitude    quaternion kinematics of quadrotor_dynamics.py:122,129 + the spacecraft
//               Euler equation (nx = 7; the reference has no such model)
//   cartpole    diffmpc/dynamics/cartpole_dynamics.py:36-80
//   integrator  diffmpc/dynamics/integrators.py:20-71
#pragma once
#include "dual.cuh"
#include "../../include/dmpc.h"

template <int MODEL>
struct ModelDims;
template <>
struct ModelDims<DMPC_MODEL_LINEAR> {
  static constexpr int NX = DMPC_MAX_NX, NU = DMPC_MAX_NU;
};
template <>
struct ModelDims<DMPC_MODEL_QUADROTOR> {
  static constexpr int NX = 13, NU = 4;
};
template <>
struct ModelDims<DMPC_MODEL_SPACECRAFT> {
  static constexpr int NX = 3, NU = 3;
};
template <>
struct ModelDims<DMPC_MODEL_ATTITUDE> {
  static constexpr int NX = 7, NU = 3;
};
template <>
struct ModelDims<DMPC_MODEL_CARTPOLE> {
  static constexpr int NX = 4, NU = 1;
};

__host__ __device__ inline int model_param_count(int model, int nx, int nu) {
  switch (model) {
    case DMPC_MODEL_LINEAR: return nx * nx + nx * nu + nx;
    case DMPC_MODEL_QUADROTOR: return 10;
    case DMPC_MODEL_SPACECRAFT: return 3;
    case DMPC_MODEL_ATTITUDE: return 3;
    case DMPC_MODEL_CARTPOLE: return 4;
  }
  return -1;
}

__host__ __device__ inline bool model_dims_ok(int model, int nx, int nu) {
  switch (model) {
    case DMPC_MODEL_LINEAR: return nx >= 1 && nx <= DMPC_MAX_NX && nu >= 1 && nu <= DMPC_MAX_NU;
    case DMPC_MODEL_QUADROTOR: return nx == 13 && nu == 4;
    case DMPC_MODEL_SPACECRAFT: return nx == 3 && nu == 3;
    case DMPC_MODEL_ATTITUDE: return nx == 7 && nu == 3;
    case DMPC_MODEL_CARTPOLE: return nx == 4 && nu == 1;
  }
  return false;
}

// 3x3 inverse by the adjugate (the reference calls jnp.linalg.inv; equal up to rounding)
template <class T>
__device__ __forceinline__ void inv3(const T* m, T* r) {
  T c00 = m[4] * m[8] - m[5] * m[7];
  T c01 = m[5] * m[6] - m[3] * m[8];
  T c02 = m[3] * m[7] - m[4] * m[6];
  T det = m[0] * c00 + m[1] * c01 + m[2] * c02;
  T id = 1.0 / det;
  r[0] = c00 * id;
  r[1] = (m[2] * m[7] - m[1] * m[8]) * id;
  r[2] = (m[1] * m[5] - m[2] * m[4]) * id;
  r[3] = c01 * id;
  r[4] = (m[0] * m[8] - m[2] * m[6]) * id;
  r[5] = (m[2] * m[3] - m[0] * m[5]) * id;
  r[6] = c02 * id;
  r[7] = (m[1] * m[6] - m[0] * m[7]) * id;
  r[8] = (m[0] * m[4] - m[1] * m[3]) * id;
}

template <class T, int MODEL>
struct StateDot;

template <class T>
struct StateDot<T, DMPC_MODEL_LINEAR> {
  __device__ static void eval(int nx, int nu, const T* x, const T* u, const T* p, T* xd) {
    const T* A = p;
    const T* B = p + nx * nx;
    const T* b = B + nx * nu;
    for (int i = 0; i < nx; ++i) {
      T a = 0.0;
      for (int j = 0; j < nx; ++j) a = a + A[i * nx + j] * x[j];
      T c = 0.0;
      for (int j = 0; j < nu; ++j) c = c + B[i * nu + j] * u[j];
      xd[i] = a + c + b[i];
    }
  }
};

template <class T>
struct StateDot<T, DMPC_MODEL_QUADROTOR> {
  __device__ static void eval(int, int, const T* x, const T* u, const T* p, T* xd) {
    const double g = 9.81;
    T J[9], Ji[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) J[k] = p[1 + k];
    inv3(J, Ji);
    T m = p[0];
    T qw = x[6], qx = x[7], qy = x[8], qz = x[9];
    T nrm = dsqrt(qw * qw + qx * qx + qy * qy + qz * qz);
    qw = qw / nrm;
    qx = qx / nrm;
    qy = qy / nrm;
    qz = qz / nrm;
    T wx = x[10], wy = x[11], wz = x[12];
    T f = u[0];
    // R e3 (third column of the rotation matrix, quadrotor_dynamics.py:63-68)
    T qw2 = qw * qw, qx2 = qx * qx, qy2 = qy * qy, qz2 = qz * qz;
    T re0 = 2.0 * (qx * qz + qw * qy);
    T re1 = 2.0 * (qy * qz - qw * qx);
    T re2 = qw2 - qx2 - qy2 + qz2;
    T fm = f / m;
    xd[0] = x[3];
    xd[1] = x[4];
    xd[2] = x[5];
    xd[3] = fm * re0;
    xd[4] = fm * re1;
    xd[5] = fm * re2 - g;
    // 0.5 q_left(q) [0; w]
    xd[6] = 0.5 * (-(qx * wx) - qy * wy - qz * wz);
    xd[7] = 0.5 * (qw * wx - qz * wy + qy * wz);
    xd[8] = 0.5 * (qz * wx + qw * wy - qx * wz);
    xd[9] = 0.5 * (-(qy * wx) + qx * wy + qw * wz);
    // J^-1 (S(J w) w + tau),  S(a) b = a x b
    T a0 = J[0] * wx + J[1] * wy + J[2] * wz;
    T a1 = J[3] * wx + J[4] * wy + J[5] * wz;
    T a2 = J[6] * wx + J[7] * wy + J[8] * wz;
    T c0 = a1 * wz - a2 * wy + u[1];
    T c1 = a2 * wx - a0 * wz + u[2];
    T c2 = a0 * wy - a1 * wx + u[3];
    xd[10] = Ji[0] * c0 + Ji[1] * c1 + Ji[2] * c2;
    xd[11] = Ji[3] * c0 + Ji[4] * c1 + Ji[5] * c2;
    xd[12] = Ji[6] * c0 + Ji[7] * c1 + Ji[8] * c2;
  }
};

template <class T>
struct StateDot<T, DMPC_MODEL_SPACECRAFT> {
  __device__ static void eval(int, int, const T* x, const T* u, const T* p, T* xd) {
    T J0 = p[0], J1 = p[1], J2 = p[2];
    T h0 = J0 * x[0], h1 = J1 * x[1], h2 = J2 * x[2];
    // omega_cross @ (J omega) = omega x (J omega)
    T c0 = x[1] * h2 - x[2] * h1;
    T c1 = x[2] * h0 - x[0] * h2;
    T c2 = x[0] * h1 - x[1] * h0;
    xd[0] = (1.0 / J0) * (u[0] - c0);
    xd[1] = (1.0 / J1) * (u[1] - c1);
    xd[2] = (1.0 / J2) * (u[2] - c2);
  }
};

template <class T>
struct StateDot<T, DMPC_MODEL_ATTITUDE> {
  __device__ static void eval(int, int, const T* x, const T* u, const T* p, T* xd) {
    T qw = x[0], qx = x[1], qy = x[2], qz = x[3];
    T nrm = dsqrt(qw * qw + qx * qx + qy * qy + qz * qz);
    qw = qw / nrm;
    qx = qx / nrm;
    qy = qy / nrm;
    qz = qz / nrm;
    T wx = x[4], wy = x[5], wz = x[6];
    xd[0] = 0.5 * (-(qx * wx) - qy * wy - qz * wz);
    xd[1] = 0.5 * (qw * wx - qz * wy + qy * wz);
    xd[2] = 0.5 * (qz * wx + qw * wy - qx * wz);
    xd[3] = 0.5 * (-(qy * wx) + qx * wy + qw * wz);
    T J0 = p[0], J1 = p[1], J2 = p[2];
    T h0 = J0 * wx, h1 = J1 * wy, h2 = J2 * wz;
    T c0 = wy * h2 - wz * h1;
    T c1 = wz * h0 - wx * h2;
    T c2 = wx * h1 - wy * h0;
    xd[4] = (1.0 / J0) * (u[0] - c0);
    xd[5] = (1.0 / J1) * (u[1] - c1);
    xd[6] = (1.0 / J2) * (u[2] - c2);
  }
};

template <class T>
struct StateDot<T, DMPC_MODEL_CARTPOLE> {
  __device__ static void eval(int, int, const T* x, const T* u, const T* p, T* xd) {
    T m_c = p[0], m_p = p[1], length = p[2], g = p[3];
    T total = m_c + m_p;
    T pml = m_p * length;
    T s = dsin(x[2]), c = dcos(x[2]);
    T temp = (u[0] + pml * x[3] * x[3] * s) / total;
    T theta_acc = (g * s - c * temp) / (length * (4.0 / 3.0 - (m_p * c * c) / total));
    T x_acc = temp - pml * theta_acc * c / total;
    xd[0] = x[1];
    xd[1] = x_acc;
    xd[2] = x[3];
    xd[3] = theta_acc;
  }
};

// One integration step x_next = F(x, u) (integrators.py:20-71).  Like the
// reference, the Euler step is always formed first.
template <class T, int MODEL>
__device__ void predict_next_state(int scheme, double dt, int nx, int nu, const T* x, const T* u,
                                   const T* p, T* xn) {
  constexpr int MX = ModelDims<MODEL>::NX;
  // fixed-size models have nx == MX: compile-time trip counts keep the arrays in registers
  T k[MX], tmp[MX], acc[MX];
  StateDot<T, MODEL>::eval(nx, nu, x, u, p, k);
  for (int i = 0; i < (MODEL != DMPC_MODEL_LINEAR ? MX : nx); ++i) xn[i] = x[i] + dt * k[i];
  if (scheme == DMPC_MIDPOINT) {
    for (int i = 0; i < (MODEL != DMPC_MODEL_LINEAR ? MX : nx); ++i) tmp[i] = x[i] + 0.5 * dt * k[i];
    StateDot<T, MODEL>::eval(nx, nu, tmp, u, p, acc);
    for (int i = 0; i < (MODEL != DMPC_MODEL_LINEAR ? MX : nx); ++i) xn[i] = x[i] + dt * acc[i];
  } else if (scheme == DMPC_RK4) {
    for (int i = 0; i < (MODEL != DMPC_MODEL_LINEAR ? MX : nx); ++i) {
      acc[i] = k[i];
      tmp[i] = x[i] + 0.5 * dt * k[i];
    }
    StateDot<T, MODEL>::eval(nx, nu, tmp, u, p, k);  // k2
    for (int i = 0; i < (MODEL != DMPC_MODEL_LINEAR ? MX : nx); ++i) {
      acc[i] = acc[i] + 2.0 * k[i];
      tmp[i] = x[i] + 0.5 * dt * k[i];
    }
    StateDot<T, MODEL>::eval(nx, nu, tmp, u, p, k);  // k3
    for (int i = 0; i < (MODEL != DMPC_MODEL_LINEAR ? MX : nx); ++i) {
      acc[i] = acc[i] + 2.0 * k[i];
      tmp[i] = x[i] + dt * k[i];
    }
    StateDot<T, MODEL>::eval(nx, nu, tmp, u, p, k);  // k4
    for (int i = 0; i < (MODEL != DMPC_MODEL_LINEAR ? MX : nx); ++i) xn[i] = x[i] + ((1.0 / 6.0) * (acc[i] + k[i])) * dt;
  }
}
