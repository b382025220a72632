// gsofa_io.cpp -- binary CSR files: the parsed form of the reference's three
// ASCII .dat files, so a matrix is parsed once and then loaded at file-read
// speed.
//
// Layout (little-endian):
//   bytes  0..7   magic "GSOFACSR"
//          8..11  version (1)
//         12..15  n (int32)
//         16..23  nnz (int64)
//         24..31  checksum of the payload (see payload_checksum)
//         32..63  zero
//   then  beg[n], end[n], col[nnz] as int32: row v is col[beg[v] .. end[v]),
//   exactly as in the .dat files (rows need not be contiguous or sorted).
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "gsofa_host.h"

using namespace gsofa::host;

namespace {

constexpr char kMagic[8] = {'G', 'S', 'O', 'F', 'A', 'C', 'S', 'R'};
constexpr uint32_t kVersion = 1;
constexpr size_t kHeader = 64;

// Fletcher-style pair of running sums over the payload's 32-bit words
// (mod 2^64): catches truncation, swapped blocks and flipped bits.
struct Checksum {
    uint64_t s1 = 0, s2 = 0;
    void add(const int32_t* p, size_t count) {
        for (size_t i = 0; i < count; i++) {
            s1 += (uint32_t)p[i];
            s2 += s1;
        }
    }
    uint64_t value() const { return s2 ^ (s1 << 32) ^ (s1 >> 32); }
};

uint64_t payload_checksum(int32_t n, int64_t nnz, const int32_t* beg, const int32_t* end,
                          const int32_t* col) {
    Checksum c;
    c.add(beg, (size_t)n);
    c.add(end, (size_t)n);
    c.add(col, (size_t)nnz);
    return c.value();
}

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) fclose(f);
    }
};

// Reads and checks the header; leaves the file positioned at the payload.
int read_header(FILE* f, int32_t* n, int64_t* nnz, uint64_t* sum) {
    unsigned char h[kHeader];
    if (fread(h, 1, kHeader, f) != kHeader) return GSOFA_ERR_IO;
    if (memcmp(h, kMagic, 8) != 0) return GSOFA_ERR_IO;
    uint32_t ver;
    memcpy(&ver, h + 8, 4);
    if (ver != kVersion) return GSOFA_ERR_UNSUPPORTED;
    memcpy(n, h + 12, 4);
    memcpy(nnz, h + 16, 8);
    memcpy(sum, h + 24, 8);
    if (*n < 0 || *nnz < 0 || *nnz > INT32_MAX) return GSOFA_ERR_IO;
    // the file must hold exactly the payload the header announces
    const long long want = (long long)kHeader + 4ll * (2ll * *n + *nnz);
    if (fseek(f, 0, SEEK_END) != 0) return GSOFA_ERR_IO;
    if (ftell(f) != want) return GSOFA_ERR_IO;
    if (fseek(f, (long)kHeader, SEEK_SET) != 0) return GSOFA_ERR_IO;
    return GSOFA_OK;
}

int read_payload(FILE* f, int32_t n, int64_t nnz, uint64_t sum, int32_t* beg, int32_t* end,
                 int32_t* col) {
    if (fread(beg, 4, (size_t)n, f) != (size_t)n) return GSOFA_ERR_IO;
    if (fread(end, 4, (size_t)n, f) != (size_t)n) return GSOFA_ERR_IO;
    if (fread(col, 4, (size_t)nnz, f) != (size_t)nnz) return GSOFA_ERR_IO;
    if (payload_checksum(n, nnz, beg, end, col) != sum) return GSOFA_ERR_IO;
    return GSOFA_OK;
}

}  // namespace

extern "C" {

int gsofa_write_csr_binary(const char* path, int32_t n, int64_t nnz, const int32_t* row_begin,
                           const int32_t* row_end, const int32_t* col) {
    if (!path || n < 0 || nnz < 0 || nnz > INT32_MAX) return GSOFA_ERR_ARG;
    if ((n > 0 && (!row_begin || !row_end)) || (nnz > 0 && !col)) return GSOFA_ERR_ARG;
    unsigned char h[kHeader] = {};
    memcpy(h, kMagic, 8);
    memcpy(h + 8, &kVersion, 4);
    memcpy(h + 12, &n, 4);
    memcpy(h + 16, &nnz, 8);
    const uint64_t sum = payload_checksum(n, nnz, row_begin, row_end, col);
    memcpy(h + 24, &sum, 8);
    // write to a temporary name, then rename: a reader never sees half a file
    const std::string tmp = std::string(path) + ".tmp";
    File f;
    f.f = fopen(tmp.c_str(), "wb");
    if (!f.f) return GSOFA_ERR_IO;
    bool ok = fwrite(h, 1, kHeader, f.f) == kHeader;
    ok = ok && fwrite(row_begin, 4, (size_t)n, f.f) == (size_t)n;
    ok = ok && fwrite(row_end, 4, (size_t)n, f.f) == (size_t)n;
    ok = ok && fwrite(col, 4, (size_t)nnz, f.f) == (size_t)nnz;
    ok = (fclose(f.f) == 0) && ok;
    f.f = nullptr;
    if (!ok || rename(tmp.c_str(), path) != 0) {
        remove(tmp.c_str());
        return GSOFA_ERR_IO;
    }
    return GSOFA_OK;
}

int gsofa_read_csr_binary(const char* path, int32_t* n, int64_t* nnz, int32_t* row_begin,
                          int32_t* row_end, int32_t* col) {
    if (!path || !n || !nnz) return GSOFA_ERR_ARG;
    File f;
    f.f = fopen(path, "rb");
    if (!f.f) return GSOFA_ERR_IO;
    int32_t fn = 0;
    int64_t fnnz = 0;
    uint64_t sum = 0;
    int rc = read_header(f.f, &fn, &fnnz, &sum);
    if (rc) return rc;
    *n = fn;
    *nnz = fnnz;
    if (!row_begin && !row_end && !col) return GSOFA_OK;  // size query
    if ((fn > 0 && (!row_begin || !row_end)) || (fnnz > 0 && !col)) return GSOFA_ERR_ARG;
    return read_payload(f.f, fn, fnnz, sum, row_begin, row_end, col);
}

int gsofa_convert_dat_to_binary(const char* beg_file, const char* end_file, const char* csr_file,
                                const char* out_path) {
    if (!beg_file || !end_file || !csr_file || !out_path) return GSOFA_ERR_ARG;
    int32_t n = 0;
    int64_t nnz = 0;
    std::vector<int32_t> beg, end, col;
    int rc = parse_dat_files(nullptr, beg_file, end_file, csr_file, &n, &nnz, &beg, &end, &col);
    if (rc) return rc;
    return gsofa_write_csr_binary(out_path, n, nnz, beg.data(), end.data(), col.data());
}

int gsofa_load_csr_binary(gsofa_ctx* ctx, const char* path, gsofa_matrix** out) {
    if (!ctx || !path || !out) return GSOFA_ERR_ARG;
    *out = nullptr;
    File f;
    f.f = fopen(path, "rb");
    if (!f.f) return set_err(ctx, GSOFA_ERR_IO, "cannot read %s", path);
    int32_t n = 0;
    int64_t nnz = 0;
    uint64_t sum = 0;
    int rc = read_header(f.f, &n, &nnz, &sum);
    if (rc) return set_err(ctx, rc, "%s: not a version-1 binary CSR file of consistent size", path);
    // one buffer: beg | end | col
    std::vector<int32_t> buf(2 * (size_t)n + (size_t)nnz + 1);
    int32_t* beg = buf.data();
    int32_t* end = beg + n;
    int32_t* col = end + n;
    rc = read_payload(f.f, n, nnz, sum, beg, end, col);
    if (rc) return set_err(ctx, rc, "%s: truncated or checksum mismatch", path);
    return gsofa_load_csr(ctx, n, nnz, beg, end, col, out);
}

}  // extern "C"
