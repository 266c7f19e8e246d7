/*
 * Drop-in replacement for GAMERA-OP's ghost-fill library
 * (src/boundary_conditions.c) when the step runs on the GPU.
 *
 * The problem's boundary_conditions() hook (src/problem.h:5-12) keeps calling
 * the same gas_bc_* / gem_bc_* functions (src/common.h:18-87); here each call
 * records which fill the problem asked for on that face instead of touching
 * host memory.  Like the reference functions, a call only takes effect on a
 * face without a neighbouring domain (MPI_PROC_NULL).  The recorded kinds
 * go into the gop_desc of the device instance, whose ghost-fill kernels apply
 * the same index formulas as the reference library.
 */
#include <mpi.h>

#include "common.h"
#include "config.h"
#include "setup_mpi.h"

char gop_gas_bc[6] = {'n', 'n', 'n', 'n', 'n', 'n'};
char gop_gem_bc[6] = {'n', 'n', 'n', 'n', 'n', 'n'};

void gop_bc_record_begin(void) {
  for (int f = 0; f < 6; f++) {
    gop_gas_bc[f] = 'n';
    gop_gem_bc[f] = 'n';
  }
}

static void gop_note(char *tab, int axis, int side, char kind) {
  int nbr = side == 0 ? nbr_low[axis] : nbr_high[axis];
  if (nbr == MPI_PROC_NULL) tab[2 * axis + side] = kind;
}

#define GOP_BC_FACE(fam, tab, kind, letter, ax, axis, sd, side) \
  void fam##_bc_##kind##_##ax##_##sd(void) { gop_note(tab, axis, side, letter); }

#define GOP_BC_KIND(fam, tab, kind, letter)             \
  GOP_BC_FACE(fam, tab, kind, letter, i, 0, low, 0)     \
  GOP_BC_FACE(fam, tab, kind, letter, i, 0, high, 1)    \
  GOP_BC_FACE(fam, tab, kind, letter, j, 1, low, 0)     \
  GOP_BC_FACE(fam, tab, kind, letter, j, 1, high, 1)    \
  GOP_BC_FACE(fam, tab, kind, letter, k, 2, low, 0)     \
  GOP_BC_FACE(fam, tab, kind, letter, k, 2, high, 1)

GOP_BC_KIND(gas, gop_gas_bc, symmetric, 's')
GOP_BC_KIND(gas, gop_gas_bc, reflective, 'r')
GOP_BC_KIND(gas, gop_gas_bc, fixed, 'f')
GOP_BC_KIND(gas, gop_gas_bc, extrapolated, 'e')
GOP_BC_KIND(gas, gop_gas_bc, none, 'n')
GOP_BC_KIND(gem, gop_gem_bc, symmetric, 's')
GOP_BC_KIND(gem, gop_gem_bc, reflective, 'r')
GOP_BC_KIND(gem, gop_gem_bc, fixed, 'f')
GOP_BC_KIND(gem, gop_gem_bc, extrapolated, 'e')
GOP_BC_KIND(gem, gop_gem_bc, none, 'n')

/* the pole fills of spherical grids (src/spherical/spherical_boundary.c,
 * theta faces only) */
void gas_bc_pole_j_low(void) { gop_note(gop_gas_bc, 1, 0, 'o'); }
void gas_bc_pole_j_high(void) { gop_note(gop_gas_bc, 1, 1, 'o'); }
void gem_bc_pole_j_low(void) { gop_note(gop_gem_bc, 1, 0, 'o'); }
void gem_bc_pole_j_high(void) { gop_note(gop_gem_bc, 1, 1, 'o'); }
