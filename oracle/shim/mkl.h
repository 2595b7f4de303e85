// The two MKL symbols the reference uses, declared for the oracle's pardiso_64
// stand-in (oracle/pardiso_shim.cpp).  Oracle build of the reference only.
#pragma once
#include <cstdint>
typedef long long MKL_INT64;
extern "C" void pardiso_64(void*, const MKL_INT64*, const MKL_INT64*, const MKL_INT64*,
                           const MKL_INT64*, const MKL_INT64*, const void*, const MKL_INT64*,
                           const MKL_INT64*, MKL_INT64*, const MKL_INT64*, MKL_INT64*,
                           const MKL_INT64*, void*, void*, MKL_INT64*);
extern "C" void mkl_set_num_threads(int);
