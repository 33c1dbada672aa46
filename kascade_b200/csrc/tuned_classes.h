// Size-class table: mean ruler spacing, chains per thread and chase block
// size for instances of at most KS_TUNED_MAX[i] elements.  Written by
// kascade_b200/autotune.py from measurements on the GPU named below; the
// library starts every context with it.  The single-call spacings of the
// two largest classes (32 and 48) were re-measured on the write-free level 0
// (`bench.py --n 2^26 / 2^27 / 2^28 --spacing ...`).
#pragma once
#define KS_TUNED_GPU "NVIDIA B200"
#define KS_TUNED_COUNT 8
#define KS_TUNED_MAX {1024ull, 8192ull, 65536ull, 524288ull, 4194304ull, 33554432ull, 134217728ull, ~0ull}
#define KS_TUNED_SPACING {4u, 6u, 6u, 4u, 6u, 12u, 24u, 96u}
#define KS_TUNED_SPACING_SINGLE {48u, 6u, 12u, 12u, 24u, 32u, 32u, 48u}
#define KS_TUNED_CHAINS {1u, 1u, 1u, 1u, 1u, 1u, 4u, 4u}
#define KS_TUNED_BLOCK {256u, 128u, 128u, 512u, 512u, 512u, 512u, 512u}
