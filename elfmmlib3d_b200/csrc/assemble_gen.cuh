// assemble_gen.cuh -- GENERATED by gen_assemble.py; do not edit by hand.
#pragma once
// included from tri_integrals.cuh (needs EFMM_HD)
namespace efmm {
// Local-frame single/double layer displacement and symmetric
// strain from the R/B tables; pair_eval (tri_integrals.cuh) rotates and scales.
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
