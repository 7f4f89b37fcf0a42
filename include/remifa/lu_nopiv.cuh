// Same file name as the reference's src/lu_nopiv.cuh (remifa::lu_nopiv_panel).
// With -I include/remifa -I include, code written against the reference
// compiles unchanged against the header-only drop-in over liblu_b200.so.
#pragma once
#include "../remifa_shim.hxx"
