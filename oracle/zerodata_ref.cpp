// C-ABI harness around the reference's own ZeroData (search/fast_mertens_enum.cpp:27-277) --
// TEST INFRASTRUCTURE ONLY.
//
// The Makefile compiles this file with -DMB_ENUM_SRC="<the reference checkout>/search/
// fast_mertens_enum.cpp": the reference source is #included as it lies (its main() renamed so it
// does not clash), nothing of it is copied here.  The wrappers below only call its
// ZeroData::load (the zeros.bin reader and the precomputed cos/sin grids, :40-106),
// ZeroData::fast_screen (the two-stage FP32 cosine-table leaf screen, :108-142) and
// ZeroData::polish (the five-stage hit polish, :145-276), so tests and the fixture generator can
// pin this repository's restatements and GPU kernels to the reference's decisions and values.
// Only tests/ and the fixture generator load the resulting oracle/_ref/libzerodata_ref.so.
#define main mertens_enum_main_unused
#include MB_ENUM_SRC
#undef main

#include <cstdint>

extern "C" {

// Load a zeros.bin file (search/path1_build_zeros_100k.py layout); null on failure.  The table
// must hold at least 15,000 zeros: polish()'s fourth stage reads that many (:245-250).
void *zd_load(const char *path) {
    ZeroData *z = new ZeroData();
    if (!z->load(path)) {
        delete z;
        return nullptr;
    }
    return z;
}

void zd_free(void *h) { delete static_cast<ZeroData *>(h); }

int zd_n_zeros(const void *h) { return static_cast<const ZeroData *>(h)->n_zeros; }

// pass[i] = fast_screen(x_i) for the leaves x_i = x_hi[i] 2^64 + x_lo[i] (x = floor(y 2^30)).
void zd_fast_screen(const void *h, int64_t n, const uint64_t *x_lo, const uint64_t *x_hi, uint8_t *pass) {
    const ZeroData *z = static_cast<const ZeroData *>(h);
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t i = 0; i < n; ++i) {
        const unsigned __int128 x = ((unsigned __int128)x_hi[i] << 64) | x_lo[i];
        pass[i] = z->fast_screen(x) ? 1 : 0;
    }
}

// (h_out[i], dy_out[i]) = polish(x_i), the reference's best h and its offset dy from y_i.
void zd_polish(const void *h, int64_t n, const uint64_t *x_lo, const uint64_t *x_hi, double *h_out,
               double *dy_out) {
    const ZeroData *z = static_cast<const ZeroData *>(h);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t i = 0; i < n; ++i) {
        const unsigned __int128 x = ((unsigned __int128)x_hi[i] << 64) | x_lo[i];
        const std::pair<double, double> r = z->polish(x);
        h_out[i] = r.first;
        dy_out[i] = r.second;
    }
}

}  // extern "C"
