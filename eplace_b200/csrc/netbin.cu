// netbin.cu -- the engine's binary netlist file: the arrays of ep_netlist as
// they lie in memory, so a reader maps the file and points an ep_netlist at
// it without parsing (the Bookshelf text parser, Parser/parser.cpp:44-819,
// is the slow and lossy step of the reference's I/O; its .pl writer prints
// coordinates with %.0f).
//
// Layout (little-endian):
//   0   char[8]  "EPNETBN1"
//   8   uint32   version (1)
//   12  uint32   number of arrays (18)
//   16  int32    num_nodes, num_terminals, num_nets, num_rows, num_pins
//   36  float    common_row_height, target_density
//   44  int32    bins (0 = the reference's rule)
//   48  uint64   offset of each array from the start of the file (18 x 8 bytes),
//                every array starting on a 64-byte boundary, in this order:
//                node_w node_h node_cx node_cy (float, num_nodes)
//                term_llx term_lly term_w term_h (float, num_terminals)
//                term_is_ni (uint8, num_terminals)
//                net_start (int32, num_nets + 1) pin_owner (int32, num_pins)
//                pin_dx pin_dy (float, num_pins)
//                row_llx row_lly row_urx row_h row_site_w (float, num_rows;
//                the site width is not part of ep_netlist: the C writer
//                stores 1, the Bookshelf default)
// Host code only; no CUDA call.
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "eplace_gpu.h"

namespace {

constexpr char kMagic[8] = {'E', 'P', 'N', 'E', 'T', 'B', 'N', '1'};
constexpr uint32_t kVersion = 1;
constexpr int kArrays = 18;
constexpr size_t kHeader = 48 + 8 * kArrays;

struct NetbinFile {
    void *base = nullptr;
    size_t size = 0;
};

// (element size, element count) of array k for the given counts.
void array_shape(int k, const int32_t c[5], size_t &esz, size_t &count) {
    const int32_t nn = c[0], nt = c[1], nnet = c[2], nr = c[3], np = c[4];
    static const int kind[kArrays] = {0, 0, 0, 0, 1, 1, 1, 1, 2, 3, 4, 4, 4, 5, 5, 5, 5, 5};
    switch (kind[k]) {
        case 0: esz = 4; count = (size_t)nn; break;
        case 1: esz = 4; count = (size_t)nt; break;
        case 2: esz = 1; count = (size_t)nt; break;
        case 3: esz = 4; count = (size_t)nnet + 1; break;
        case 4: esz = 4; count = (size_t)np; break;
        default: esz = 4; count = (size_t)nr; break;
    }
}

size_t align64(size_t x) { return (x + 63) & ~(size_t)63; }

}  // namespace

extern "C" {

ep_status ep_netbin_write(const char *path, const ep_netlist *nl, float target_density, int32_t bins) try {
    if (!path || !nl || nl->num_nodes < 0 || nl->num_terminals < 0 || nl->num_nets < 0 || nl->num_rows < 0)
        return EP_ERR_ARG;
    if (nl->num_nets > 0 && !nl->net_start) return EP_ERR_ARG;
    const int32_t np = nl->num_nets > 0 ? nl->net_start[nl->num_nets] : 0;
    const int32_t c[5] = {nl->num_nodes, nl->num_terminals, nl->num_nets, nl->num_rows, np};
    std::vector<uint8_t> ni;
    const uint8_t *term_ni = nl->term_is_ni;
    if (!term_ni) {
        ni.assign(nl->num_terminals, 0);
        term_ni = ni.data();
    }
    const int32_t zero_start = 0;
    std::vector<float> site(nl->num_rows, 1.0f);
    const void *src[kArrays] = {nl->node_w, nl->node_h, nl->node_cx, nl->node_cy, nl->term_llx, nl->term_lly,
                                nl->term_w, nl->term_h, term_ni, nl->num_nets > 0 ? nl->net_start : &zero_start,
                                nl->pin_owner, nl->pin_dx, nl->pin_dy, nl->row_llx, nl->row_lly, nl->row_urx,
                                nl->row_h, site.data()};
    uint64_t off[kArrays];
    size_t pos = align64(kHeader);
    for (int k = 0; k < kArrays; k++) {
        size_t esz, n;
        array_shape(k, c, esz, n);
        off[k] = pos;
        pos = align64(pos + esz * n);
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) return EP_ERR_ARG;
    std::vector<uint8_t> head(align64(kHeader), 0);
    std::memcpy(&head[0], kMagic, 8);
    const uint32_t meta[2] = {kVersion, (uint32_t)kArrays};
    std::memcpy(&head[8], meta, 8);
    std::memcpy(&head[16], c, 20);
    const float fl[2] = {nl->common_row_height, target_density};
    std::memcpy(&head[36], fl, 8);
    std::memcpy(&head[44], &bins, 4);
    std::memcpy(&head[48], off, 8 * kArrays);
    bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
    size_t at = head.size();
    static const uint8_t pad[64] = {0};
    for (int k = 0; ok && k < kArrays; k++) {
        size_t esz, n;
        array_shape(k, c, esz, n);
        if (at < off[k]) {
            ok = std::fwrite(pad, 1, off[k] - at, f) == off[k] - at;
            at = off[k];
        }
        if (n == 0) continue;
        if (!src[k]) {
            ok = false;
            break;
        }
        ok = std::fwrite(src[k], esz, n, f) == n;
        at += esz * n;
    }
    ok = std::fclose(f) == 0 && ok;
    return ok ? EP_OK : EP_ERR_ARG;
} catch (const std::bad_alloc &) {
    return EP_ERR_NOMEM;
}

ep_status ep_netbin_open(const char *path, ep_netlist *nl, float *target_density, int32_t *bins,
                         void **handle) {
    if (!path || !nl || !handle) return EP_ERR_ARG;
    *handle = nullptr;
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) return EP_ERR_ARG;
    struct stat st;
    if (fstat(fd, &st) != 0 || (size_t)st.st_size < kHeader) {
        ::close(fd);
        return EP_ERR_ARG;
    }
    void *base = mmap(nullptr, (size_t)st.st_size, PROT_READ, MAP_PRIVATE, fd, 0);
    ::close(fd);
    if (base == MAP_FAILED) return EP_ERR_ARG;
    const uint8_t *b = (const uint8_t *)base;
    uint32_t meta[2];
    int32_t c[5];
    float fl[2];
    int32_t bn;
    uint64_t off[kArrays];
    std::memcpy(meta, b + 8, 8);
    std::memcpy(c, b + 16, 20);
    std::memcpy(fl, b + 36, 8);
    std::memcpy(&bn, b + 44, 4);
    std::memcpy(off, b + 48, 8 * kArrays);
    bool ok = std::memcmp(b, kMagic, 8) == 0 && meta[0] == kVersion && meta[1] == (uint32_t)kArrays;
    for (int k = 0; ok && k < 5; k++) ok = c[k] >= 0;
    for (int k = 0; ok && k < kArrays; k++) {
        size_t esz, n;
        array_shape(k, c, esz, n);
        ok = off[k] % 64 == 0 && off[k] + esz * n <= (size_t)st.st_size;
    }
    if (ok && c[2] > 0) {
        const int32_t *ns = (const int32_t *)(b + off[9]);
        ok = ns[0] == 0 && ns[c[2]] == c[4];
    }
    if (!ok) {
        munmap(base, (size_t)st.st_size);
        return EP_ERR_ARG;
    }
    auto F = [&](int k) { return (const float *)(b + off[k]); };
    nl->num_nodes = c[0];
    nl->num_terminals = c[1];
    nl->num_nets = c[2];
    nl->num_rows = c[3];
    nl->node_w = F(0);
    nl->node_h = F(1);
    nl->node_cx = F(2);
    nl->node_cy = F(3);
    nl->term_llx = F(4);
    nl->term_lly = F(5);
    nl->term_w = F(6);
    nl->term_h = F(7);
    nl->term_is_ni = b + off[8];
    nl->net_start = (const int32_t *)(b + off[9]);
    nl->pin_owner = (const int32_t *)(b + off[10]);
    nl->pin_dx = F(11);
    nl->pin_dy = F(12);
    nl->row_llx = F(13);
    nl->row_lly = F(14);
    nl->row_urx = F(15);
    nl->row_h = F(16);
    nl->common_row_height = fl[0];
    if (target_density) *target_density = fl[1];
    if (bins) *bins = bn;
    NetbinFile *h = new (std::nothrow) NetbinFile;
    if (!h) {
        munmap(base, (size_t)st.st_size);
        return EP_ERR_NOMEM;
    }
    h->base = base;
    h->size = (size_t)st.st_size;
    *handle = h;
    return EP_OK;
}

void ep_netbin_close(void *handle) {
    NetbinFile *h = (NetbinFile *)handle;
    if (!h) return;
    if (h->base) munmap(h->base, h->size);
    delete h;
}

}  // extern "C"
