/* CPU oracle for OpenLB's collide-and-stream — TEST INFRASTRUCTURE ONLY.
 * See olb_oracle.h for scope and the parity pin.  Build: oracle/Makefile
 * (-O2 -ffp-contract=off so every multiply and add rounds as written). */
#include "olb_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* D3Q19: descriptor/definition/common.h:135-163 */
static const int c19[19][3] = {
  { 0, 0, 0},
  {-1, 0, 0}, { 0,-1, 0}, { 0, 0,-1}, {-1,-1, 0}, {-1, 1, 0}, {-1, 0,-1},
  {-1, 0, 1}, { 0,-1,-1}, { 0,-1, 1},
  { 1, 0, 0}, { 0, 1, 0}, { 0, 0, 1}, { 1, 1, 0}, { 1,-1, 0}, { 1, 0, 1},
  { 1, 0,-1}, { 0, 1, 1}, { 0, 1,-1}
};
static const int opp19[19] = {0, 10, 11, 12, 13, 14, 15, 16, 17, 18, 1, 2, 3, 4, 5, 6, 7, 8, 9};
static const int w19[19][2] = {
  {1, 3},
  {1, 18}, {1, 18}, {1, 18}, {1, 36}, {1, 36}, {1, 36}, {1, 36}, {1, 36}, {1, 36},
  {1, 18}, {1, 18}, {1, 18}, {1, 36}, {1, 36}, {1, 36}, {1, 36}, {1, 36}, {1, 36}
};

/* D3Q27: descriptor/definition/common.h:328-364 */
static const int c27[27][3] = {
  { 0, 0, 0},
  {-1, 0, 0}, { 0,-1, 0}, { 0, 0,-1}, {-1,-1, 0}, {-1, 1, 0}, {-1, 0,-1},
  {-1, 0, 1}, { 0,-1,-1}, { 0,-1, 1}, {-1,-1,-1}, {-1,-1, 1}, {-1, 1,-1}, {-1, 1, 1},
  { 1, 0, 0}, { 0, 1, 0}, { 0, 0, 1}, { 1, 1, 0}, { 1,-1, 0}, { 1, 0, 1},
  { 1, 0,-1}, { 0, 1, 1}, { 0, 1,-1}, { 1, 1, 1}, { 1, 1,-1}, { 1,-1, 1}, { 1,-1,-1}
};
static const int opp27[27] = {0, 14, 15, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26,
                              1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13};
static const int w27[27][2] = {
  {8, 27},
  {2, 27}, {2, 27}, {2, 27}, {1, 54}, {1, 54}, {1, 54}, {1, 54}, {1, 54}, {1, 54},
  {1, 216}, {1, 216}, {1, 216}, {1, 216},
  {2, 27}, {2, 27}, {2, 27}, {1, 54}, {1, 54}, {1, 54}, {1, 54}, {1, 54}, {1, 54},
  {1, 216}, {1, 216}, {1, 216}, {1, 216}
};

static int get_tables(int q, const int (**c)[3], const int** opp)
{
  if (q == 19) { *c = c19; *opp = opp19; return 0; }
  if (q == 27) { *c = c27; *opp = opp27; return 0; }
  return -1;
}

/* Fraction::as<T>() = T(num) / T(den)  utilities/fraction.h:58-62 */
static int weight_num(int q, int i) { return q == 19 ? w19[i][0] : w27[i][0]; }
static int weight_den(int q, int i) { return q == 19 ? w19[i][1] : w27[i][1]; }

#define REAL float
#define SFX f32
#include "olb_oracle_impl.inc"
#undef REAL
#undef SFX

#define REAL double
#define SFX f64
#include "olb_oracle_impl.inc"
#undef REAL
#undef SFX

int oracle_descriptor(int q, int32_t* c, int32_t* opposite, double* w)
{
  const int (*cc)[3];
  const int* oo;
  if (get_tables(q, &cc, &oo) != 0) {
    return -1;
  }
  for (int i = 0; i < q; ++i) {
    for (int d = 0; d < 3; ++d) {
      c[3 * i + d] = cc[i][d];
    }
    opposite[i] = oo[i];
    w[i] = (double)weight_num(q, i) / (double)weight_den(q, i);
  }
  return 0;
}
