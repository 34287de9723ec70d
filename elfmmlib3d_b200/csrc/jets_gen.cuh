// jets_gen.cuh -- GENERATED by gen_jets.py; do not edit by hand.
#pragma once
// included from jets.cuh (needs EFMM_HD)
namespace efmm {
EFMM_HD void jet3_mul(const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ z) {
  z[0] = x[0] * y[0];
  z[1] = x[0] * y[1] + x[1] * y[0];
  z[2] = x[0] * y[2] + x[2] * y[0];
  z[3] = x[0] * y[3] + x[3] * y[0];
  z[4] = x[0] * y[4] + x[1] * y[1] + x[4] * y[0];
  z[5] = x[0] * y[5] + x[1] * y[2] + x[2] * y[1] + x[5] * y[0];
  z[6] = x[0] * y[6] + x[1] * y[3] + x[3] * y[1] + x[6] * y[0];
  z[7] = x[0] * y[7] + x[2] * y[2] + x[7] * y[0];
  z[8] = x[0] * y[8] + x[2] * y[3] + x[3] * y[2] + x[8] * y[0];
  z[9] = x[0] * y[9] + x[3] * y[3] + x[9] * y[0];
  z[10] = x[0] * y[10] + x[1] * y[4] + x[4] * y[1] + x[10] * y[0];
  z[11] = x[0] * y[11] + x[1] * y[5] + x[2] * y[4] + x[4] * y[2] + x[5] * y[1] + x[11] * y[0];
  z[12] = x[0] * y[12] + x[1] * y[6] + x[3] * y[4] + x[4] * y[3] + x[6] * y[1] + x[12] * y[0];
  z[13] = x[0] * y[13] + x[1] * y[7] + x[2] * y[5] + x[5] * y[2] + x[7] * y[1] + x[13] * y[0];
  z[14] = x[0] * y[14] + x[1] * y[8] + x[2] * y[6] + x[3] * y[5] + x[5] * y[3] + x[6] * y[2] + x[8] * y[1] + x[14] * y[0];
  z[15] = x[0] * y[15] + x[1] * y[9] + x[3] * y[6] + x[6] * y[3] + x[9] * y[1] + x[15] * y[0];
  z[16] = x[0] * y[16] + x[2] * y[7] + x[7] * y[2] + x[16] * y[0];
  z[17] = x[0] * y[17] + x[2] * y[8] + x[3] * y[7] + x[7] * y[3] + x[8] * y[2] + x[17] * y[0];
  z[18] = x[0] * y[18] + x[2] * y[9] + x[3] * y[8] + x[8] * y[3] + x[9] * y[2] + x[18] * y[0];
  z[19] = x[0] * y[19] + x[3] * y[9] + x[9] * y[3] + x[19] * y[0];
}
// Accumulate one edge's contribution to the in-plane table entries.
EFMM_HD void tables_edge(const double* __restrict__ L1, const double* __restrict__ Lr,
                         double mx, double my, double* __restrict__ R, double* __restrict__ B) {
  B[1] += (1.0) * mx * Lr[0];
  R[1] += (1.0) * mx * L1[0];
  B[2] += (1.0) * my * Lr[0];
  R[2] += (1.0) * my * L1[0];
  B[4] += (-1.0) * mx * Lr[1];
  R[4] += (-1.0) * mx * L1[1];
  B[5] += (-1.0) * mx * Lr[2];
  R[5] += (-1.0) * mx * L1[2];
  B[6] += (-1.0) * mx * Lr[3];
  R[6] += (-1.0) * mx * L1[3];
  B[7] += (-1.0) * my * Lr[2];
  R[7] += (-1.0) * my * L1[2];
  B[8] += (-1.0) * my * Lr[3];
  R[8] += (-1.0) * my * L1[3];
  B[10] += (2.0) * mx * Lr[4];
  B[11] += (1.0) * mx * Lr[5];
  B[12] += (1.0) * mx * Lr[6];
  B[13] += (2.0) * mx * Lr[7];
  B[14] += (1.0) * mx * Lr[8];
  B[15] += (2.0) * mx * Lr[9];
  B[16] += (2.0) * my * Lr[7];
  B[17] += (1.0) * my * Lr[8];
  B[18] += (2.0) * my * Lr[9];
  B[20] += (-6.0) * mx * Lr[10];
  B[21] += (-2.0) * mx * Lr[11];
  B[22] += (-2.0) * mx * Lr[12];
  B[23] += (-2.0) * mx * Lr[13];
  B[24] += (-1.0) * mx * Lr[14];
  B[25] += (-2.0) * mx * Lr[15];
  B[26] += (-6.0) * mx * Lr[16];
  B[27] += (-2.0) * mx * Lr[17];
  B[28] += (-2.0) * mx * Lr[18];
  B[29] += (-6.0) * mx * Lr[19];
  B[30] += (-6.0) * my * Lr[16];
  B[31] += (-2.0) * my * Lr[17];
  B[32] += (-2.0) * my * Lr[18];
  B[33] += (-6.0) * my * Lr[19];
}
// Local-frame single/double layer displacement and (unsymmetrised x2)
// displacement gradient from the tables (see assemble_local in tri_integrals.cuh).
EFMM_HD void assemble_gen(const double* __restrict__ R, const double* __restrict__ B,
    double rlam, double rmu, double c1, const double* ssl, const double* sdl,
    bool dosl, bool dodl, bool dostrain, double* __restrict__ ul, double* __restrict__ el) {
  for (int i = 0; i < 3; i++) ul[i] = 0.0;
  for (int i = 0; i < 6; i++) el[i] = 0.0;
  if (dosl) {
    const double s0 = ssl[0], s1 = ssl[1], s2 = ssl[2];
    ul[0] += s0 * (-c1 * B[4] + 2.0 * R[0]) + s1 * (-c1 * B[5]) + s2 * (-c1 * B[6]);
    ul[1] += s0 * (-c1 * B[5]) + s1 * (-c1 * B[7] + 2.0 * R[0]) + s2 * (-c1 * B[8]);
    ul[2] += s0 * (-c1 * B[6]) + s1 * (-c1 * B[8]) + s2 * (-c1 * B[9] + 2.0 * R[0]);
    if (dostrain) {
      el[0] += s0 * (-c1 * B[10] + (R[1] + R[1])) + s1 * (-c1 * B[11]) + s2 * (-c1 * B[12]);
      el[1] += s0 * (-c1 * B[13]) + s1 * (-c1 * B[16] + (R[2] + R[2])) + s2 * (-c1 * B[17]);
      el[2] += s0 * (-c1 * B[15]) + s1 * (-c1 * B[18]) + s2 * (-c1 * B[19] + (R[3] + R[3]));
      el[3] += s0 * (-c1 * B[11] + (R[2])) + s1 * (-c1 * B[13] + (R[1])) + s2 * (-c1 * B[14]);
      el[4] += s0 * (-c1 * B[12] + (R[3])) + s1 * (-c1 * B[14]) + s2 * (-c1 * B[15] + (R[1]));
      el[5] += s0 * (-c1 * B[14]) + s1 * (-c1 * B[17] + (R[3])) + s2 * (-c1 * B[18] + (R[2]));
    }
  }
  if (dodl) {
    const double s0 = sdl[0], s1 = sdl[1], s2 = sdl[2];
    ul[0] += s0 * (rmu * ((-c1 * B[12] + 2.0 * R[3]) + (-c1 * B[12]))) + s1 * (rmu * ((-c1 * B[14]) + (-c1 * B[14]))) + s2 * (rmu * ((-c1 * B[15]) + (-c1 * B[15])) + rlam * ((-c1 * B[10] + 2.0 * R[1]) + (-c1 * B[13]) + (-c1 * B[15])));
    ul[1] += s0 * (rmu * ((-c1 * B[14]) + (-c1 * B[14]))) + s1 * (rmu * ((-c1 * B[17] + 2.0 * R[3]) + (-c1 * B[17]))) + s2 * (rmu * ((-c1 * B[18]) + (-c1 * B[18])) + rlam * ((-c1 * B[11]) + (-c1 * B[16] + 2.0 * R[2]) + (-c1 * B[18])));
    ul[2] += s0 * (rmu * ((-c1 * B[15]) + (-c1 * B[15] + 2.0 * R[1]))) + s1 * (rmu * ((-c1 * B[18]) + (-c1 * B[18] + 2.0 * R[2]))) + s2 * (rmu * ((-c1 * B[19] + 2.0 * R[3]) + (-c1 * B[19] + 2.0 * R[3])) + rlam * ((-c1 * B[12]) + (-c1 * B[17]) + (-c1 * B[19] + 2.0 * R[3])));
    if (dostrain) {
      el[0] += s0 * (rmu * ((-c1 * B[22] + 2.0 * R[6]) + (-c1 * B[22]))) + s1 * (rmu * ((-c1 * B[24]) + (-c1 * B[24]))) + s2 * (rmu * ((-c1 * B[25]) + (-c1 * B[25])) + rlam * ((-c1 * B[20] + 2.0 * R[4]) + (-c1 * B[23]) + (-c1 * B[25])));
      el[1] += s0 * (rmu * ((-c1 * B[27]) + (-c1 * B[27]))) + s1 * (rmu * ((-c1 * B[31] + 2.0 * R[8]) + (-c1 * B[31]))) + s2 * (rmu * ((-c1 * B[32]) + (-c1 * B[32])) + rlam * ((-c1 * B[23]) + (-c1 * B[30] + 2.0 * R[7]) + (-c1 * B[32])));
      el[2] += s0 * (rmu * ((-c1 * B[29]) + (-c1 * B[29] + 2.0 * R[6]))) + s1 * (rmu * ((-c1 * B[33]) + (-c1 * B[33] + 2.0 * R[8]))) + s2 * (rmu * ((-c1 * B[34] + 2.0 * R[9]) + (-c1 * B[34] + 2.0 * R[9])) + rlam * ((-c1 * B[25]) + (-c1 * B[32]) + (-c1 * B[34] + 2.0 * R[9])));
      el[3] += s0 * 0.5 * (rmu * ((-c1 * B[24] + 2.0 * R[8]) + (-c1 * B[24])) + rmu * ((-c1 * B[24]) + (-c1 * B[24]))) + s1 * 0.5 * (rmu * ((-c1 * B[27]) + (-c1 * B[27])) + rmu * ((-c1 * B[27] + 2.0 * R[6]) + (-c1 * B[27]))) + s2 * 0.5 * (rmu * ((-c1 * B[28]) + (-c1 * B[28])) + rlam * ((-c1 * B[21] + 2.0 * R[5]) + (-c1 * B[26]) + (-c1 * B[28])) + rmu * ((-c1 * B[28]) + (-c1 * B[28])) + rlam * ((-c1 * B[21]) + (-c1 * B[26] + 2.0 * R[5]) + (-c1 * B[28])));
      el[4] += s0 * 0.5 * (rmu * ((-c1 * B[25] + 2.0 * R[9]) + (-c1 * B[25])) + rmu * ((-c1 * B[25]) + (-c1 * B[25] + 2.0 * R[4]))) + s1 * 0.5 * (rmu * ((-c1 * B[28]) + (-c1 * B[28])) + rmu * ((-c1 * B[28]) + (-c1 * B[28] + 2.0 * R[5]))) + s2 * 0.5 * (rmu * ((-c1 * B[29]) + (-c1 * B[29])) + rlam * ((-c1 * B[22] + 2.0 * R[6]) + (-c1 * B[27]) + (-c1 * B[29])) + rmu * ((-c1 * B[29] + 2.0 * R[6]) + (-c1 * B[29] + 2.0 * R[6])) + rlam * ((-c1 * B[22]) + (-c1 * B[27]) + (-c1 * B[29] + 2.0 * R[6])));
      el[5] += s0 * 0.5 * (rmu * ((-c1 * B[28]) + (-c1 * B[28])) + rmu * ((-c1 * B[28]) + (-c1 * B[28] + 2.0 * R[5]))) + s1 * 0.5 * (rmu * ((-c1 * B[32] + 2.0 * R[9]) + (-c1 * B[32])) + rmu * ((-c1 * B[32]) + (-c1 * B[32] + 2.0 * R[7]))) + s2 * 0.5 * (rmu * ((-c1 * B[33]) + (-c1 * B[33])) + rlam * ((-c1 * B[24]) + (-c1 * B[31] + 2.0 * R[8]) + (-c1 * B[33])) + rmu * ((-c1 * B[33] + 2.0 * R[8]) + (-c1 * B[33] + 2.0 * R[8])) + rlam * ((-c1 * B[24]) + (-c1 * B[31]) + (-c1 * B[33] + 2.0 * R[8])));
    }
  }
}
}  // namespace efmm
