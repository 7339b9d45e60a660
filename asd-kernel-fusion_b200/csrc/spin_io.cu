// spin_io.cu -- on-disk format for spin states (host code only).
//
// The reference keeps spins only in memory; this library defines a file
// format so that runs can be checkpointed and resumed and states exchanged
// with the reference's own programs (the payload is the reference's AoS
// layout, double[nfile][N*N][3], llg_sqt_baseline.c:185, :202).
//
// Layout (little-endian):
//   bytes  0..7   magic "ASDSPIN1"
//   bytes  8..11  int32 N
//   bytes 12..15  int32 nfile
//   bytes 16..23  int64 step (time step the state belongs to)
//   bytes 24..31  double spin_len
//   bytes 32..63  reserved, zero
//   bytes 64..    nfile*N*N*3 doubles
#include <cstdint>
#include <cstdio>
#include <cstring>

#include "asd_internal.h"

namespace {
constexpr char kMagic[8] = {'A', 'S', 'D', 'S', 'P', 'I', 'N', '1'};
constexpr int kHeader = 64;

struct Header {
    char magic[8];
    int32_t N;
    int32_t nfile;
    int64_t step;
    double spin_len;
    unsigned char reserved[32];
};
static_assert(sizeof(Header) == kHeader, "header size");
}  // namespace

using namespace asd;

extern "C" {

int asd_spins_save(const char *path, int N, int nfile, long step, double spin_len,
                   const double *spin_aos) {
    if (!path || !spin_aos) return fail(ASD_ERR_INVALID, "NULL argument");
    if (N < 1 || nfile < 1) return fail(ASD_ERR_INVALID, "N=%d nfile=%d", N, nfile);
    Header h;
    std::memset(&h, 0, sizeof h);
    std::memcpy(h.magic, kMagic, 8);
    h.N = N;
    h.nfile = nfile;
    h.step = step;
    h.spin_len = spin_len;
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(ASD_ERR_INVALID, "cannot open %s for writing", path);
    const size_t n = (size_t)nfile * N * N * 3;
    const bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 && std::fwrite(spin_aos, sizeof(double), n, f) == n;
    const bool closed = std::fclose(f) == 0;
    if (!ok || !closed) return fail(ASD_ERR_INVALID, "short write to %s", path);
    return ASD_OK;
}

int asd_spins_load(const char *path, int *N, int *nfile, long *step, double *spin_len,
                   double *spin_aos, size_t capacity) {
    if (!path || !N || !nfile) return fail(ASD_ERR_INVALID, "NULL argument");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(ASD_ERR_INVALID, "cannot open %s", path);
    Header h;
    if (std::fread(&h, sizeof h, 1, f) != 1 || std::memcmp(h.magic, kMagic, 8) != 0) {
        std::fclose(f);
        return fail(ASD_ERR_INVALID, "%s is not a spin file", path);
    }
    if (h.N < 1 || h.nfile < 1 || (double)h.N * h.N * h.nfile * 3 > 4.0e9) {
        std::fclose(f);
        return fail(ASD_ERR_INVALID, "%s: bad header (N=%d nfile=%d)", path, h.N, h.nfile);
    }
    *N = h.N;
    *nfile = h.nfile;
    if (step) *step = (long)h.step;
    if (spin_len) *spin_len = h.spin_len;
    const size_t n = (size_t)h.nfile * h.N * h.N * 3;
    if (!spin_aos) {  // size query
        std::fclose(f);
        return ASD_OK;
    }
    if (capacity < n) {
        std::fclose(f);
        return fail(ASD_ERR_INVALID, "buffer holds %zu doubles, the file has %zu", capacity, n);
    }
    const size_t got = std::fread(spin_aos, sizeof(double), n, f);
    std::fclose(f);
    if (got != n) return fail(ASD_ERR_INVALID, "%s is truncated (%zu of %zu values)", path, got, n);
    return ASD_OK;
}

}  // extern "C"
