// Plain structs shared by the host planner and the CUDA kernels.
#pragma once

#include <stdint.h>

#define KATE_MAX_QUBITS 40
#define KATE_MAX_TILE 14

// Device op kinds.
#define OPK_DENSE 0  // dense 2^k x 2^k on tile bits tb[0..k-1] (bit i of local index <-> tb[i])
#define OPK_H 1      // Hadamard on tile bit tb[0], with the reference's arithmetic
#define OPK_X 2      // NOT on tile bit tb[0] where all controls are 1 (CNOT, TOFFOLI)
#define OPK_PHASE 3  // multiply by (ph_re, ph_im) where all controls are 1 (CRk)
#define OPK_DIAG 4   // multiply by table[sum_i bit_i << i], bit i from ftb[i] (tile) or fpos[i] (coset)

typedef struct {
    int32_t kind;
    int32_t k;         // dense / diag qubit count
    int32_t tb[5];     // target tile bits (dense bit order), tb[0] for H / X
    int32_t ftb[5];    // diag qubit i: tile bit, or -1 when outside the tile
    int32_t fpos[5];   // diag qubit i outside the tile: physical bit
    uint32_t tmask;    // controls inside the tile (tile-bit mask)
    uint64_t pmask;    // controls outside the tile (physical-bit mask)
    int64_t mat;       // offset into the matrix pool, in complex elements
    double ph_re, ph_im;
} DevOp;

typedef struct {
    int32_t m;          // tile bits
    int32_t nops;
    int32_t op0;        // first op index
    int32_t ncb;        // coset bits = n - m
    uint8_t tphys[16];  // physical bit of tile bit t (ascending)
    uint8_t outsrc[16]; // on store, output tile bit t takes input tile bit outsrc[t]
    uint8_t cphys[48];  // physical bits of the coset index, ascending
} DevPass;
