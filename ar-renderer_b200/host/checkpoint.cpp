// Checkpoint files of a progressive GPU render in the reference's PRCKPT02 layout
// (src/integrators/integrator.cpp:16-90, src/core/film.cpp:61-84): an 8-byte magic, the packed
// header (integrator | GPU bit, max depth, width, height, chains, scene fingerprint, seed), the
// film's FP64 XYZ accumulators (count, then values), and a length-prefixed body (for the path
// tracer: the samples per pixel already rendered). Files are written to "<path>.tmp" and renamed
// into place, so a crash never leaves a half-written checkpoint under the final name.

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/prhost_api.h"

namespace {

constexpr char kMagic[8] = {'P', 'R', 'C', 'K', 'P', 'T', '0', '2'};
constexpr size_t kHeaderBytes = 8 + 4 + 4 * 4 + 8 + 8;

void set_err(char *err, int errLen, const std::string &msg) {
    if (!err || errLen <= 0) return;
    std::snprintf(err, size_t(errLen), "%s", msg.c_str());
}

// The header exactly as the reference's BinaryWriter emits it: fields packed, native byte order.
std::vector<unsigned char> header_bytes(const prhost::CheckpointHeader &h) {
    std::vector<unsigned char> b(kHeaderBytes);
    unsigned char *p = b.data();
    auto put = [&p](const void *v, size_t n) {
        std::memcpy(p, v, n);
        p += n;
    };
    put(kMagic, 8);
    put(&h.integrator, 4);
    put(&h.maxDepth, 4);
    put(&h.width, 4);
    put(&h.height, 4);
    put(&h.chains, 4);
    put(&h.fingerprint, 8);
    put(&h.seed, 8);
    return b;
}

} // namespace

PRHOST_API int prhost_checkpoint_write(const char *path, const prhost::CheckpointHeader *header, const double *film,
                                       uint64_t filmCount, const void *body, uint64_t bodySize, char *err,
                                       int errLen) {
    if (!path || !header || (filmCount && !film) || (bodySize && !body) || header->width <= 0 ||
        header->height <= 0 || filmCount != uint64_t(header->width) * uint64_t(header->height) * 3) {
        set_err(err, errLen, "bad checkpoint arguments");
        return 1;
    }
    const std::string tmp = std::string(path) + ".tmp";
    FILE *f = std::fopen(tmp.c_str(), "wb");
    if (!f) {
        set_err(err, errLen, "cannot write checkpoint " + tmp);
        return 1;
    }
    const std::vector<unsigned char> hdr = header_bytes(*header);
    bool ok = std::fwrite(hdr.data(), 1, hdr.size(), f) == hdr.size();
    ok = ok && std::fwrite(&filmCount, sizeof(filmCount), 1, f) == 1;
    // The film in 8 MiB pieces (it can be gigabytes at 16K).
    for (uint64_t i = 0; ok && i < filmCount; i += uint64_t(1) << 20) {
        const size_t m = size_t(filmCount - i < (uint64_t(1) << 20) ? filmCount - i : (uint64_t(1) << 20));
        ok = std::fwrite(film + i, sizeof(double), m, f) == m;
    }
    ok = ok && std::fwrite(&bodySize, sizeof(bodySize), 1, f) == 1;
    ok = ok && (bodySize == 0 || std::fwrite(body, 1, size_t(bodySize), f) == bodySize);
    ok = std::fclose(f) == 0 && ok;
    if (ok) ok = std::rename(tmp.c_str(), path) == 0;
    if (!ok) {
        std::remove(tmp.c_str());
        set_err(err, errLen, std::string("failed to write checkpoint ") + path);
        return 1;
    }
    return 0;
}

PRHOST_API int prhost_checkpoint_read(const char *path, const prhost::CheckpointHeader *expected, double *film,
                                      uint64_t filmCount, void *body, uint64_t bodyCapacity, uint64_t *bodySize,
                                      char *err, int errLen) {
    if (!path || !expected || (filmCount && !film) || (bodyCapacity && !body) || !bodySize) {
        set_err(err, errLen, "bad checkpoint arguments");
        return 1;
    }
    FILE *f = std::fopen(path, "rb");
    if (!f) {
        set_err(err, errLen, std::string("cannot open checkpoint ") + path);
        return 1;
    }
    const std::vector<unsigned char> want = header_bytes(*expected);
    std::vector<unsigned char> got(want.size());
    const bool readHeader = std::fread(got.data(), 1, got.size(), f) == got.size();
    if (!readHeader || std::memcmp(got.data(), want.data(), 8) != 0) {
        std::fclose(f);
        set_err(err, errLen, std::string(path) + " is not a prender checkpoint");
        return 2;
    }
    if (std::memcmp(got.data(), want.data(), want.size()) != 0) {
        std::fclose(f);
        set_err(err, errLen, std::string(path) + " was made for a different scene, integrator, device, resolution, seed or depth");
        return 3;
    }
    uint64_t n = 0, size = 0;
    bool ok = std::fread(&n, sizeof(n), 1, f) == 1 && n == filmCount;
    for (uint64_t i = 0; ok && i < n; i += uint64_t(1) << 20) {
        const size_t m = size_t(n - i < (uint64_t(1) << 20) ? n - i : (uint64_t(1) << 20));
        ok = std::fread(film + i, sizeof(double), m, f) == m;
    }
    ok = ok && std::fread(&size, sizeof(size), 1, f) == 1 && size <= bodyCapacity;
    ok = ok && (size == 0 || std::fread(body, 1, size_t(size), f) == size);
    std::fclose(f);
    if (!ok) {
        set_err(err, errLen, std::string(path) + " is truncated or corrupt");
        return 4;
    }
    *bodySize = size;
    return 0;
}
