// Tile and schedule constants of the kernels.  The autotuner (openmm-interax-plugin_b200/tune.py) times candidate
// values on the benchmark's shapes on the GPU and records the chosen ones in openmm-interax-plugin_b200/tuning.json;
// the build passes them to the compiler as the IX_TUNE_* macros below.  The defaults here are used only when a build
// is made without that file.
#pragma once

// pair kernel: warps per thread block, queued pairs evaluated before their forces are gathered, and the minimum
// resident blocks per SM the compiler is told to fit (which bounds its registers per thread)
#ifndef IX_TUNE_PAIR_WARPS
#define IX_TUNE_PAIR_WARPS 4
#endif
#ifndef IX_TUNE_PAIR_ROUND
#define IX_TUNE_PAIR_ROUND 128
#endif
#ifndef IX_TUNE_PAIR_MIN_BLOCKS
#define IX_TUNE_PAIR_MIN_BLOCKS 8
#endif
// pair kernel: 1 = per-tile column lists for the column-force gather, 0 = found from the row masks each round
#ifndef IX_TUNE_PAIR_COLUMN_LISTS
#define IX_TUNE_PAIR_COLUMN_LISTS 0
#endif
// pair kernel: 1 = each tile's column masks formed in registers as the transpose of its row masks on every path;
// 0 = loaded from the tile list where the candidates are not filtered against the cutoff when queued (the list holds
// both, the columns the exact transpose of the rows)
#ifndef IX_TUNE_PAIR_COLUMN_TRANSPOSE
#define IX_TUNE_PAIR_COLUMN_TRANSPOSE 0
#endif
// pair kernel: 1 = two queued pairs per lane at a time on the class-table path without per-pair tests
#ifndef IX_TUNE_PAIR_ILP
#define IX_TUNE_PAIR_ILP 0
#endif
// pair kernel: largest class-pair table (bytes) staged in shared memory; larger tables are read through the cache
#ifndef IX_TUNE_PAIR_SHARED_TABLE_BYTES
#define IX_TUNE_PAIR_SHARED_TABLE_BYTES 0
#endif
// pair kernel: the most parameter classes (particles with identical pair parameters) for which it reads each pair's
// coefficients from a class-pair table (at most 256: the class is 8 bits of the flags); above, per-particle parameters
#ifndef IX_TUNE_PAIR_MAX_CLASSES
#define IX_TUNE_PAIR_MAX_CLASSES 16
#endif
// pair list: skin (nm) of the list cutoff; the list is rebuilt when a particle has moved by half of it
#ifndef IX_TUNE_PAIR_SKIN
#define IX_TUNE_PAIR_SKIN 0.1f
#endif
// three-body: skin of the site lists, the longest list the fast triple kernel takes, (B, C) pairs per round
#ifndef IX_TUNE_SITE_SKIN
#define IX_TUNE_SITE_SKIN 0.1f
#endif
#ifndef IX_TUNE_ATM_FAST
#define IX_TUNE_ATM_FAST 64
#endif
#ifndef IX_TUNE_ATM_ROUND
#define IX_TUNE_ATM_ROUND 64
#endif
// three-body: minimum resident blocks of the fast triple kernel per SM (bounds its registers per thread)
#ifndef IX_TUNE_ATM_MIN_BLOCKS
#define IX_TUNE_ATM_MIN_BLOCKS 7
#endif
// three-body: 1 = the fast kernel adds each triple's B and C forces to per-neighbor 64-bit fixed-point sums in shared
// memory (integer atomics, no rounds); 0 = it stores them per round and gathers them per neighbor
#ifndef IX_TUNE_ATM_ACCUM
#define IX_TUNE_ATM_ACCUM 0
#endif
