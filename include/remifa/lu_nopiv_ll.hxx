// Same file name as the reference's src/lu_nopiv_ll.hxx (remifa::lu_nopiv_ll and the
// lu_nopiv_ll_* wrappers).
// With -I include/remifa -I include, code written against the reference
// compiles unchanged against the header-only drop-in over liblu_b200.so.
#pragma once
#include "../remifa_shim.hxx"
