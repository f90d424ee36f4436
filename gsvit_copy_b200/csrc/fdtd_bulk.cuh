// fdtd_bulk.cuh -- TMA-staged bulk kernel (fdtd_bulk.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "fdtd_internal.h"

// tensor maps of the input field set and of the class map
struct BulkMaps {
    CUtensorMap e[3];
    CUtensorMap h[3];
    CUtensorMap cls;
};

// one CTA: own cells [j0, min(j0+15, jhi)) x [k0, min(k0+60, khi)) of planes [ib, ie)
struct BulkItem {
    int j0, k0, ib, ie, jhi, khi, inst, pad0;   // inst: plan of the item in a batched launch
};

// own rows and columns of a tile; the bulk box has 1 <= lo, hi <= res - 1 on
// every axis and its k bounds (hence k0 and khi) are multiples of 4
#define BULK_TJ 15
#define BULK_TK 60

size_t bulk_smem_bytes(int nclasses, int storage);
cudaError_t bulk_configure();
cudaError_t launch_bulk(const DevPlan &p, const BulkMaps &m, const BulkItem *items, int nitems, int *err, bool ade,
                        int npoles, int storage, cudaStream_t st);
// all items of many plans in one persistent launch of `grid` CTAs; plans and
// maps are device tables of this step's parity, indexed by BulkItem::inst
cudaError_t launch_bulk_batch(const DevPlan *plans, const BulkMaps *maps, const BulkItem *items, int nitems, int grid,
                              int ncls_layout, int *err, bool ade, int npoles, int storage, cudaStream_t st);
int bulk_make_maps(void *encode_fn, const DevPlan &p, float *const f[6], const uint8_t *cls, int cls_pitch, int storage,
                   BulkMaps *out);
