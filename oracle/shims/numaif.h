/* ORACLE shim (see numa.h). */
#ifndef ORACLE_NUMAIF_SHIM_H
#define ORACLE_NUMAIF_SHIM_H
#define MPOL_MF_STRICT (1 << 0)
#define MPOL_MF_MOVE (1 << 1)
#define MPOL_MF_MOVE_ALL (1 << 2)
#endif
