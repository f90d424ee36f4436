// fdtd_bulk.cuh -- TMA-staged tile kernels (fdtd_bulk.cu): the bulk of the grid
// and the CPML tiles around it.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fdtd_internal.h"

// tensor maps of the input field set and of the class map (box shapes of one
// tile layout)
struct BulkMaps {
    CUtensorMap e[3];
    CUtensorMap h[3];
    CUtensorMap cls;
};

// one CTA: own cells [max(j0, jlo), min(j0+TJ, jhi)) x [max(k0, klo), min(k0+TK, khi))
// of planes [ib, ie); a tile may start below its region (j0 < jlo, k0 < klo,
// even below 0): those rows and groups only supply halo values
struct BulkItem {
    int j0, k0, ib, ie, jlo, jhi, klo, khi, inst, pad0;   // inst: plan of the item in a batched launch
};

// Tile layouts: own rows (TJ) and own k cells (TK) of one CTA of 256 threads.
//  bulk  15 x 60: the interior box, where every cell takes the plain update
//        (no CPML, kappa 1, no edge rule);
//  cpxy  15 x 60: the x slabs (whole planes; kind TILE_CPX) and the y slabs
//        (kind TILE_CPY);
//  cpz   31 x 28: the z slabs between the y slabs (TILE_CPZ).
// The CPML tiles run the special path of fdtd_cpgroup.cuh (psi, kappa, zeroed
// planes, ADE-in-CPML, edges) on every group; each kind's kernel carries the
// code of the faces its tiles can meet only.  k0, klo and khi are multiples
// of 4 in every layout.
#define BULK_TJ 15
#define BULK_TK 60
#define CPXY_TJ 15
#define CPXY_TK 60
#define CPZ_TJ 31
#define CPZ_TK 28

enum { TILE_BULK = 0, TILE_CPX = 1, TILE_CPY = 2, TILE_CPZ = 3, NTILE = 4 };
// faces a CPML tile kind can meet (its kernel carries only their code)
enum { CPF_X = 1, CPF_Y = 2, CPF_Z = 4 };

size_t tile_smem_bytes(int kind, int nclasses, int storage);
cudaError_t bulk_configure();
// `stall` > 0 (tests only): every CTA also waits, at most `stall` polls, on an
// mbarrier nothing arrives on, so that its bounded-wait error path runs
cudaError_t launch_tiles(int kind, const DevPlan &p, const BulkMaps &m, const BulkItem *items, int nitems, int *err,
                         bool ade, int npoles, int storage, int stall, cudaStream_t st);
// all bulk items of many plans in one persistent launch of `grid` CTAs (bulk
// layout); plans and maps are device tables of this step's parity, indexed by
// BulkItem::inst
cudaError_t launch_bulk_batch(const DevPlan *plans, const BulkMaps *maps, const BulkItem *items, int nitems, int grid,
                              int ncls_layout, int *err, bool ade, int npoles, int storage, cudaStream_t st);
// the tiles of many plans, one CTA per item: plans and maps (of `kind`'s
// layout) are device tables of this step's parity, indexed by BulkItem::inst
cudaError_t launch_tiles_batch(int kind, const DevPlan *plans, const BulkMaps *maps, const BulkItem *items, int nitems,
                               int ncls_layout, int *err, bool ade, int npoles, int storage, cudaStream_t st);
int tile_make_maps(int kind, void *encode_fn, const DevPlan &p, float *const f[6], const uint8_t *cls, int cls_pitch,
                   int storage, BulkMaps *out);
