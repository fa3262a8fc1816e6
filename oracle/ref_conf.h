/* Test infrastructure only: configuration for compiling the reference CPU
 * B+tree (open-harmonia/src) as the parity oracle.  Never linked into the
 * product library.
 *
 * This file is pre-included (g++ -include) ahead of every reference source.
 * Defining the include guard of open-harmonia/src/conf_for_bpt.h:1-3 makes the
 * reference skip that file's `#define TREE_32` (open-harmonia/src/conf_for_bpt.h:7),
 * so key_t/value_t become `long long` with Max_Key = LLONG_MAX
 * (open-harmonia/src/bpt.h:25-27), the 64-bit build the paper measures.
 * AVX_ALL keeps the reference's default AVX2 child search
 * (open-harmonia/src/conf_for_bpt.h:10, open-harmonia/src/bpt.h:81-85,
 * open-harmonia/src/avx.cpp:2-54). */
#define CONF_FOR_BPT_H
#define AVX_ALL
