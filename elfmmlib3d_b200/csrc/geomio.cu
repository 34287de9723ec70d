// geomio.cu -- flat-triangle geometry I/O (host code): the Cart3D ".tri"
// format the reference reads and writes (src/trilib.f:59-168: atrireadchk,
// atriwrite), its four-way refinement (matlab/atrirefine.m) and the
// triangle arrays the FMM entry points take (src/trilib.f:192-240: buildtri,
// triangle_norm, triangle_area).
//
// Format: a line "nverts nfaces", then nverts vertices (three reals each),
// then nfaces vertex-index triples (1-based), all free-format whitespace
// separated.  Arrays follow the reference's Fortran layout: verts(3,nverts),
// ifaces(3,nfaces), triangle(3,3,ntri), centroids(3,ntri), trinorm(3,ntri).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include "../../include/elfmm3d_b200.h"

namespace {

// next whitespace-separated token of the file as a double; false at the end
// of the file or on a token that is not a number
bool next_num(FILE* f, double* v) {
  char buf[128];
  if (fscanf(f, "%127s", buf) != 1) return false;
  // Fortran list-directed input also accepts exponents written with D
  for (char* c = buf; *c; c++)
    if (*c == 'd' || *c == 'D') *c = 'e';
  char* end = nullptr;
  *v = strtod(buf, &end);
  return end && *end == '\0' && end != buf;
}

bool next_int(FILE* f, int* v) {
  double d;
  if (!next_num(f, &d) || d != std::floor(d) || std::fabs(d) > 2147483647.0) return false;
  *v = (int)d;
  return true;
}

}  // namespace

extern "C" int efmm_tri_read(const char* path, double* verts, int lv, int* nverts, int* ifaces, int li,
                             int* nfaces) {
  if (!path || !nverts || !nfaces) return 16;
  FILE* f = fopen(path, "r");
  if (!f) return 1;
  int nv = 0, nf = 0;
  if (!next_int(f, &nv) || !next_int(f, &nf) || nv < 0 || nf < 0) {
    fclose(f);
    return 4;
  }
  *nverts = nv;
  *nfaces = nf;
  // sizes only (lv = li = 0) or arrays too short: the reference's ier 2 / 3
  if (lv < nv) {
    fclose(f);
    return 2;
  }
  if (li < nf) {
    fclose(f);
    return 3;
  }
  for (long long k = 0; k < 3LL * nv; k++)
    if (!next_num(f, &verts[k])) {
      fclose(f);
      return 4;
    }
  for (long long k = 0; k < 3LL * nf; k++)
    if (!next_int(f, &ifaces[k]) || ifaces[k] < 1 || ifaces[k] > nv) {
      fclose(f);
      return 4;
    }
  fclose(f);
  return 0;
}

extern "C" int efmm_tri_write(const char* path, const double* verts, int nverts, const int* ifaces, int nfaces) {
  if (!path || nverts < 0 || nfaces < 0) return 16;
  FILE* f = fopen(path, "w");
  if (!f) return 1;
  fprintf(f, " %d %d\n", nverts, nfaces);
  // 17 significant digits: the vertices read back bit for bit
  for (int j = 0; j < nverts; j++)
    fprintf(f, " %.16e %.16e %.16e\n", verts[3 * j], verts[3 * j + 1], verts[3 * j + 2]);
  for (int j = 0; j < nfaces; j++) fprintf(f, " %7d %7d %7d\n", ifaces[3 * j], ifaces[3 * j + 1], ifaces[3 * j + 2]);
  const int bad = ferror(f);
  return (fclose(f) != 0 || bad) ? 1 : 0;
}

extern "C" int efmm_tri_refine(const double* verts, int nverts, const int* ifaces, int nfaces, double* verts1,
                               int* ifaces1) {
  if (nverts < 0 || nfaces < 0) return 16;
  for (long long k = 0; k < 3LL * nfaces; k++)
    if (ifaces[k] < 1 || ifaces[k] > nverts) return 16;
  // vertices: the originals, then the midpoints of edges 1-2, 2-3 and 3-1 of
  // every face (one block per edge, face order; shared edges not merged)
  for (long long k = 0; k < 3LL * nverts; k++) verts1[k] = verts[k];
  for (int e = 0; e < 3; e++)
    for (int j = 0; j < nfaces; j++) {
      const int a = ifaces[3 * j + e] - 1, b = ifaces[3 * j + (e + 1) % 3] - 1;
      double* m = verts1 + 3 * ((long long)nverts + (long long)e * nfaces + j);
      for (int c = 0; c < 3; c++) m[c] = 0.5 * (verts[3 * a + c] + verts[3 * b + c]);
    }
  // faces: the three corner triangles (one block per corner), then the
  // middle ones; m12, m23, m31 are the face's midpoints (1-based)
  for (int j = 0; j < nfaces; j++) {
    const int v1 = ifaces[3 * j], v2 = ifaces[3 * j + 1], v3 = ifaces[3 * j + 2];
    const int m12 = nverts + j + 1, m23 = nverts + nfaces + j + 1, m31 = nverts + 2 * nfaces + j + 1;
    const int tri[4][3] = {{v1, m12, m31}, {v2, m23, m12}, {v3, m31, m23}, {m12, m23, m31}};
    for (int q = 0; q < 4; q++)
      for (int c = 0; c < 3; c++) ifaces1[3 * ((long long)q * nfaces + j) + c] = tri[q][c];
  }
  return 0;
}

extern "C" int efmm_tri_build(const double* verts, int nverts, int ntri, const int* itrivert, double* triangle,
                              double* centroids, double* trinorm, double* triarea) {
  if (nverts < 0 || ntri < 0) return 16;
  for (long long k = 0; k < 3LL * ntri; k++)
    if (itrivert[k] < 1 || itrivert[k] > nverts) return 16;
  for (int t = 0; t < ntri; t++) {
    double v[3][3];
    for (int i = 0; i < 3; i++)
      for (int c = 0; c < 3; c++) v[i][c] = verts[3 * (itrivert[3 * t + i] - 1) + c];
    for (int i = 0; i < 3; i++)
      for (int c = 0; c < 3; c++) triangle[9 * (long long)t + 3 * i + c] = v[i][c];
    if (centroids)
      for (int c = 0; c < 3; c++) centroids[3 * (long long)t + c] = (v[0][c] + v[1][c] + v[2][c]) / 3;
    // unit normal of the positively oriented triangle from (v2 - v1) x (v3 - v2),
    // area from |(v2 - v1) x (v3 - v1)| / 2: the reference's two formulas
    // (src/trilib.f:245-318), so that both round as the reference's do
    auto cross = [](const double* a, const double* b, double* n) {
      n[0] = a[1] * b[2] - a[2] * b[1];
      n[1] = a[2] * b[0] - a[0] * b[2];
      n[2] = a[0] * b[1] - a[1] * b[0];
    };
    const double x[3] = {v[1][0] - v[0][0], v[1][1] - v[0][1], v[1][2] - v[0][2]};
    const double y[3] = {v[2][0] - v[1][0], v[2][1] - v[1][1], v[2][2] - v[1][2]};
    const double z[3] = {v[2][0] - v[0][0], v[2][1] - v[0][1], v[2][2] - v[0][2]};
    double n[3], m[3];
    cross(x, y, n);
    cross(x, z, m);
    const double len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (trinorm)
      for (int c = 0; c < 3; c++) trinorm[3 * (long long)t + c] = n[c] / len;
    if (triarea) triarea[t] = 0.5 * std::sqrt(m[0] * m[0] + m[1] * m[1] + m[2] * m[2]);
  }
  return 0;
}
