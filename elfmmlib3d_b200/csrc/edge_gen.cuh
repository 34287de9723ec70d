// edge_gen.cuh -- GENERATED by gen_edge.py; do not edit by hand.
#pragma once
// included from tri_integrals.cuh (needs EFMM_HD)
namespace efmm {
// Add one edge's contribution to the in-plane table entries R (|a| = 1, 2),
// B (|a| = 2..4) and to sh = d_h (d_xx + d_yy) int 1/r.  L1: edge-frame
// derivatives of int 1/r dl (|b| <= 2), Lr: of int r dl (1 <= |b| <= 3),
// both indexed by jidx(u, v, h); (tx, ty): unit edge tangent.
EFMM_HD void edge_tables_gen(double tx, double ty, const double* __restrict__ L1,
                             const double* __restrict__ Lr, double* __restrict__ R,
                             double* __restrict__ B, double& sh) {
  const double q0 = Lr[1]*ty - Lr[2]*tx;
  const double q1 = L1[1]*ty - L1[2]*tx;
  const double q2 = (tx*tx);
  const double q3 = (ty*ty);
  const double q4 = tx*ty;
  const double q5 = 2*q4;
  const double q6 = Lr[5]*q5;
  const double q7 = Lr[4]*q3 + Lr[7]*q2 - q6;
  const double q8 = Lr[6]*ty - Lr[8]*tx;
  const double q9 = (tx*tx*tx);
  const double q10 = (ty*ty*ty);
  const double q11 = q2*ty;
  const double q12 = Lr[11]*q11;
  const double q13 = q3*tx;
  const double q14 = Lr[13]*q13;
  const double q15 = Lr[11]*q13;
  const double q16 = Lr[13]*q11;
  const double q17 = Lr[14]*q5;
  const double q18 = Lr[10]*q10 - Lr[16]*q9 - 3*q15 + 3*q16;
  const double q19 = Lr[12]*q3 + Lr[17]*q2 - q17;
  const double q20 = Lr[15]*ty - Lr[18]*tx;
  R[1] += L1[0]*ty;
  R[2] += -L1[0]*tx;
  B[4] += -ty*(Lr[1]*tx + Lr[2]*ty);
  R[4] += -ty*(L1[1]*tx + L1[2]*ty);
  B[5] += -q0*ty;
  R[5] += -q1*ty;
  B[6] += -Lr[3]*ty;
  R[6] += -L1[3]*ty;
  B[7] += q0*tx;
  R[7] += q1*tx;
  B[8] += Lr[3]*tx;
  R[8] += L1[3]*tx;
  B[10] += ty*(Lr[4]*q2 + Lr[7]*q3 + q6);
  B[11] += ty*(Lr[4]*q4 - Lr[5]*q2 + Lr[5]*q3 - Lr[7]*q4);
  B[12] += ty*(Lr[6]*tx + Lr[8]*ty);
  B[13] += q7*ty;
  B[14] += q8*ty;
  B[15] += Lr[9]*ty;
  B[16] += -q7*tx;
  B[17] += -q8*tx;
  B[18] += -Lr[9]*tx;
  B[20] += -ty*(Lr[10]*q9 + Lr[16]*q10 + 3*q12 + 3*q14);
  B[21] += -ty*(Lr[10]*q11 - Lr[11]*q9 + Lr[13]*q10 - Lr[16]*q13 + 2*q15 - 2*q16);
  B[22] += -ty*(Lr[12]*q2 + Lr[17]*q3 + q17);
  B[23] += -ty*(Lr[10]*q13 + Lr[11]*q10 + Lr[13]*q9 + Lr[16]*q11 - 2*q12 - 2*q14);
  B[24] += -ty*(Lr[12]*q4 - Lr[14]*q2 + Lr[14]*q3 - Lr[17]*q4);
  B[25] += -ty*(Lr[15]*tx + Lr[18]*ty);
  B[26] += -q18*ty;
  B[27] += -q19*ty;
  B[28] += -q20*ty;
  B[29] += -Lr[19]*ty;
  B[30] += q18*tx;
  B[31] += q19*tx;
  B[32] += q20*tx;
  B[33] += Lr[19]*tx;
  sh += -tx*(L1[6]*ty - L1[8]*tx) + ty*(L1[6]*tx + L1[8]*ty);
}
}  // namespace efmm
