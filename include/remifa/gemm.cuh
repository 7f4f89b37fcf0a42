// Same file name as the reference's src/gemm.cuh (remifa::gemmex and the
// CublasImpl / CutlassImpl / TC / FP tags).
// With -I include/remifa -I include, code written against the reference
// compiles unchanged against the header-only drop-in over liblu_b200.so.
#pragma once
#include "../remifa_shim.hxx"
