/* ORACLE shim: a one-node stand-in for the libnuma calls made by the
   reference (src/wavemoth.c:297-329, :416-493, :517, :644).  Node 0 owns
   every CPU in the process affinity mask; allocation is plain malloc. */
#ifndef ORACLE_NUMA_SHIM_H
#define ORACLE_NUMA_SHIM_H
#include <stddef.h>
struct bitmask { unsigned long size; unsigned long *maskp; };
struct bitmask *numa_allocate_nodemask(void);
struct bitmask *numa_allocate_cpumask(void);
void numa_free_nodemask(struct bitmask *b);
void numa_free_cpumask(struct bitmask *b);
struct bitmask *numa_get_run_node_mask(void);
struct bitmask *numa_get_membind(void);
void numa_set_membind(struct bitmask *b);
int numa_bitmask_isbitset(const struct bitmask *b, unsigned int n);
struct bitmask *numa_bitmask_setbit(struct bitmask *b, unsigned int n);
struct bitmask *numa_bitmask_clearbit(struct bitmask *b, unsigned int n);
struct bitmask *numa_bitmask_clearall(struct bitmask *b);
unsigned int numa_bitmask_nbytes(struct bitmask *b);
int numa_max_node(void);
int numa_node_to_cpus(int node, struct bitmask *mask);
void *numa_alloc_onnode(size_t size, int node);
void numa_free(void *mem, size_t size);
int numa_move_pages(int pid, unsigned long count, void **pages,
                    const int *nodes, int *status, int flags);
#endif
