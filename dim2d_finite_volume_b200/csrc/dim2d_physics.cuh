// dim2d_physics.cuh -- DIM (van der Waals + Korteweg) physics for the
// sm_100a kernels: per-node primitives and the face flux in a frame
// (n = face normal, t = tangential) so one routine serves x- and y-faces.
//
// Reference formulas (paths relative to the reference project root):
//   primitives   src/physical_models/dim2d/dim2d_prim_module.f:242-289,
//                392-453 (pressure), 515-613 (temperatures), 1056-1155
//   face fluxes  src/physical_models/dim2d/dim2d_fluxes_module.f:103-1649
//   operators    src/sd_operators/mattsson_operators/sd_operators_class.f
//                :160-1039 and sd_operators_fd_module.f:71-153
//
// Evaluation differs from the reference only by rounding: primitives are
// computed once per node instead of once per operator call, products such
// as rho*u*u use the node velocity, and divisions by dx use 1/dx.
#pragma once
#include <cuda_runtime.h>

namespace dim2d {

// Physical constants (dim2d_parameters.f:146-199) and their derived
// coefficients, computed once on the host.
struct DimConst {
  double re, we, pr, cv_r, viscous_r;
  double ire;        // 1/Re        (dim2d_fluxes_module.f:210)
  double iwe;        // 1/We        (dim2d_fluxes_module.f:212)
  double ipr;        // 1/Pr        (dim2d_fluxes_module.f:1285)
  double irepr;      // 1/(Re*Pr)   (dim2d_fluxes_module.f:1385)
  double c15cv;      // 1.5/cv_r    (dim2d_fluxes_module.f:691)
  double c3cv;       // 3/cv_r      (dim2d_prim_module.f:433)
  double two_mu;     // 2+viscous_r (dim2d_fluxes_module.f:636)
  double c38cv;      // 3/(8 cv_r): temperature from Tcl (wall_xy_equilibrium_module.f:476)
  int gravity_ac;
  double gravity;
};

// Per-node primitive quantities used by the flux formulas.
struct NodePrim {
  double u, v;   // velocity_x/y           (prim :242-289)
  double p;      // classical_pressure     (prim :425-453)
  double tcl;    // classical_temperature_eff (prim :515-544)
  double cp;     // capillarity_pressure 1/(3-rho) (prim :1056-1071)
};

__host__ __device__ __forceinline__ NodePrim node_prim(double r, double mx, double my, double e,
                                                       const DimConst& k) {
  NodePrim o;
  const double ir = 1.0 / r;
  o.u = mx * ir;
  o.v = my * ir;
  o.cp = 1.0 / (3.0 - r);
  // W = E - rho|u|^2/2 + 3 rho^2 ; P = 3/((3-rho) cv_r) W - 3 rho^2 ; Tcl = W/rho
  const double w = e - 0.5 * r * (o.u * o.u + o.v * o.v) + 3.0 * (r * r);
  o.p = k.c3cv * o.cp * w - 3.0 * (r * r);
  o.tcl = ir * w;
  return o;
}

// capillarity_temperature_eff with centred gradients (prim :582-613,
// sd_operators_fd_module.f:71-153): 0.5/rho * (drho/dx^2 + drho/dy^2).
__host__ __device__ __forceinline__ double node_tcap(double r, double rxm, double rxp, double rym,
                                                     double ryp, double hrdx, double hrdy) {
  const double gx = hrdx * (rxp - rxm);
  const double gy = hrdy * (ryp - rym);
  return 0.5 / r * (gx * gx + gy * gy);
}

// Inputs of one face flux, in the face frame.  "a" is the node on the low
// side of the face, "b" the node on the high side.  T = double for the FP64
// path, float for the face pass of the mixed-precision path.
template <typename T>
struct FaceInT {
  // conservative values: rho, momentum along n, momentum along t, energy
  T ra, rb, mna, mnb, mta, mtb, ea, eb;
  // primitives: velocity along n / t, pressure, Tcl, cp, Tcap
  T una, unb, uta, utb, pa, pb, ta, tb, ca, cb, ka, kb;
  // derivatives at the face
  T drn, drt;  // d rho / dn, d rho / dt
  T dunn;      // d u_n / dn
  T dunt;      // d u_n / dt
  T dutn;      // d u_t / dn
  T dutt;      // d u_t / dt
  T lap;       // d2 rho/dn2 + d2 rho/dt2
  T dtn;       // d Tcl / dn
  T dkn;       // d Tcap / dn
};
using FaceIn = FaceInT<double>;

// Flux coefficients in FP32 for the mixed-precision face pass.
struct FluxCoefF {
  float ire, iwe, ipr, irepr, c15cv, two_mu, viscous_r;
};
__host__ __device__ inline FluxCoefF flux_coef_f32(const DimConst& k) {
  return FluxCoefF{(float)k.ire,   (float)k.iwe,    (float)k.ipr,      (float)k.irepr,
                   (float)k.c15cv, (float)k.two_mu, (float)k.viscous_r};
}

// Face flux of the 4 conservative variables; out = {mass, momentum_n,
// momentum_t, energy}.  For an x-face n = x (dim2d_fluxes_module.f:103-117,
// 193-222, 319-348, 445-477 and the parts they call); for a y-face n = y
// (:145-159, 256-285, 382-411, 511-541), momentum_n is then momentum_y.
// DKN = false leaves out the energy term -(1/(Re Pr)) dTcap/dn of the
// capillarity part (the mixed path adds it in FP64).
template <typename T, typename K, bool DKN>
__host__ __device__ __forceinline__ void face_flux_t(const FaceInT<T>& f, const K& k, T out[4]) {
  const T h = T(0.5);
  const T avr = h * (f.ra + f.rb);
  const T avmn = h * (f.mna + f.mnb);
  const T avun = h * (f.una + f.unb);
  const T avut = h * (f.uta + f.utb);
  const T drn2 = f.drn * f.drn;
  const T drt2 = f.drt * f.drt;
  const T grad2 = drn2 + drt2;

  // mass: f(momentum_n)
  out[0] = avmn;

  // normal momentum: inviscid f(m_n u_n) + f(P); viscid (2+mu) du_n/dn +
  // mu du_t/dt; capillarity 1.5/cv f(cp) |grad rho|^2 + f(rho) lap rho
  // + 0.5 (drho_t^2 - drho_n^2)
  {
    const T inv = h * (f.mna * f.una + f.mnb * f.unb) + h * (f.pa + f.pb);
    const T vis = k.two_mu * f.dunn + k.viscous_r * f.dutt;
    const T cap = k.c15cv * (h * (f.ca + f.cb)) * grad2 + avr * f.lap + h * (-drn2 + drt2);
    out[1] = inv - k.ire * vis - k.iwe * cap;
  }
  // tangential momentum: inviscid f(m_t u_n); viscid du_n/dt + du_t/dn;
  // capillarity -drho_n drho_t
  {
    const T inv = h * (f.mta * f.una + f.mtb * f.unb);
    const T vis = f.dunt + f.dutn;
    const T cap = -f.drn * f.drt;
    out[2] = inv - k.ire * vis - k.iwe * cap;
  }
  // energy
  {
    const T inv = h * (f.ea * f.una + f.eb * f.unb) + h * (f.pa * f.una + f.pb * f.unb);
    const T vis = avun * (k.two_mu * f.dunn + k.viscous_r * f.dutt) +
                  avut * (f.dunt + f.dutn) + k.ipr * f.dtn;
    T cap = k.c15cv * (h * (f.ca * f.una + f.cb * f.unb)) * grad2 + avmn * f.lap +
            h * avun * (-drn2 + drt2) - f.drn * f.drt * avut - avr * f.drn * (f.dunn + f.dutt);
    if (DKN) cap = cap - k.irepr * f.dkn;
    out[3] = inv - k.ire * vis - k.iwe * cap;
  }
}

__host__ __device__ __forceinline__ void face_flux(const FaceIn& f, const DimConst& k,
                                                   double out[4]) {
  face_flux_t<double, DimConst, true>(f, k, out);
}

// Flux through a wall face, in the face frame (out = {mass, momentum_n,
// momentum_t, energy}); wall_xy_equilibrium_module.f:249-402 with
// :445-908.  tl = 3/(8 cv_r) temperature_eff at the interior-side node;
// dn = grid step along the normal; q = wall heat flux; q_out = +q on the
// low (S/W) side, -q on the high (N/E) side.
__host__ __device__ __forceinline__ void wall_face_flux(const FaceIn& f, double tl, double dn,
                                                        double q, double q_out,
                                                        const DimConst& k, double out[4]) {
  const double th = tl + dn * k.c38cv * k.re * k.pr * q;
  const double t_half = 0.5 * (tl + th);
  const double md_half = 0.5 * (f.ra + f.rb);
  // dim2d_prim_module.f:476-488
  const double p = 8.0 * md_half * t_half / (3.0 - md_half) - 3.0 * (md_half * md_half);
  out[0] = 0.0;
  out[1] = p - k.iwe * (md_half * f.lap + 0.5 * (-(f.drn * f.drn) + (f.drt * f.drt)));
  out[2] = -k.ire * f.dutn - k.iwe * (-f.drn * f.drt);
  out[3] = q_out;
}

// Speed of sound, dim2d_prim_module.f:1179-1215.
__host__ __device__ __forceinline__ double sound_speed(double r, double mx, double my, double e,
                                                       const DimConst& k) {
  const double u = mx / r, v = my / r;
  const double p = 3.0 / ((3.0 - r) * k.cv_r) * (e - 0.5 * r * (u * u + v * v) + 3.0 * (r * r)) -
                   3.0 * (r * r);
  const double ee = p + (r * r) * (-3.0 + 2.0 * r);
  const double b = sqrt((p + 3.0 * (r * r)) / (k.cv_r * ee));
  const double a = 1.0 / sqrt(1.0 + b * b);
  const double d = sqrt(r * r * r) * sqrt((3.0 - r) / ee);
  return sqrt(3.0) * r / (a * d);
}

}  // namespace dim2d
