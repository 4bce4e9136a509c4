// qmb_store.cu -- versioned binary table files: sectors (representatives and
// the selected irrep), stored Hamiltonians (sliced ELL) and reference-layout
// ELL tables.  They replace the reference's raw dumps (WriteArrayToFile,
// utils/print_funcs.cu:73-90, used for vals_mat.bin / ind_mat.bin at
// exact_diagonalization/HeisenbergHamAbelianSymms_CUDA.cu:149-162), which
// write bare float arrays -- indices cast to float, no sizes, no version --
// and have no reader.
//
// Layout (little-endian):
//   header, 256 bytes: magic "QMBTABLE", u32 version, u32 kind, u32 section
//     count, u32 byte-order mark 0x01020304, u64 meta[27] (kind-specific
//     scalars), u64 checksum of the section table, u64 checksum of the
//     header with this field zero;
//   section table: per section {u32 tag, u32 element bytes, u64 count,
//     u64 offset, u64 checksum of the payload};
//   payloads at 64-byte aligned offsets.
// The checksum is a 64-bit multiply-xorshift over 8-byte words, seeded with
// the length: it catches truncation and corruption, it is not a signature.
// A file is written to "<path>.tmp.<pid>" and renamed, so a reader never sees
// a half-written file under the final name.
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <memory>
#include <cstring>
#include <string>
#include <vector>

#include "qmb_ham.cuh"
#include "qmb_b200.h"

namespace qmb {
namespace {

constexpr char kMagic[8] = {'Q', 'M', 'B', 'T', 'A', 'B', 'L', 'E'};
constexpr uint32_t kVersion = 1;
constexpr uint32_t kByteOrder = 0x01020304u;
enum : uint32_t { KIND_SECTOR = 1, KIND_HAM = 2, KIND_REF_ELL = 3 };
enum : uint32_t {
    TAG_PERM = 1, TAG_REPS, TAG_CHARS,                                           // sector
    TAG_SLICE_OFF = 16, TAG_SLICE_W, TAG_COL, TAG_VAL64, TAG_VAL32, TAG_DIAG64,  // matrix
    TAG_DIAG32, TAG_T_NOPS, TAG_T_OPS, TAG_T_SCALAR,
    TAG_IND = 32, TAG_VAL, TAG_TRACK                                             // reference ELL
};

struct Header {
    char magic[8];
    uint32_t version, kind, n_sections, byte_order;
    uint64_t meta[27];
    uint64_t table_sum, header_sum;
};
static_assert(sizeof(Header) == 256, "header layout");
struct Entry {
    uint32_t tag, elem_bytes;
    uint64_t count, offset, sum;
};
static_assert(sizeof(Entry) == 32, "section entry layout");

uint64_t checksum(const void* p, size_t n) {
    const unsigned char* b = static_cast<const unsigned char*>(p);
    uint64_t h = 0xcbf29ce484222325ull ^ (uint64_t)n;
    size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        uint64_t w;
        std::memcpy(&w, b + i, 8);
        h = (h ^ w) * 0x100000001b3ull;
        h ^= h >> 29;
    }
    if (i < n) {
        uint64_t w = 0;
        std::memcpy(&w, b + i, n - i);
        h = (h ^ w) * 0x100000001b3ull;
        h ^= h >> 29;
    }
    return h;
}

uint64_t dbits(double x) {
    uint64_t u;
    std::memcpy(&u, &x, 8);
    return u;
}
double bitsd(uint64_t u) {
    double x;
    std::memcpy(&x, &u, 8);
    return x;
}

struct Section {
    uint32_t tag, elem;
    uint64_t count;
    const void* data;
};

struct File {
    FILE* f = nullptr;
    ~File() {
        if (f) std::fclose(f);
    }
};

void write_file(const char* path, uint32_t kind, const uint64_t (&meta)[27], const std::vector<Section>& secs) {
    QMB_REQUIRE(path && *path, QMB_ERR_INVALID, "empty path");
    Header hd{};
    std::memcpy(hd.magic, kMagic, 8);
    hd.version = kVersion;
    hd.kind = kind;
    hd.n_sections = (uint32_t)secs.size();
    hd.byte_order = kByteOrder;
    std::memcpy(hd.meta, meta, sizeof(hd.meta));
    std::vector<Entry> tab(secs.size());
    uint64_t off = (sizeof(Header) + sizeof(Entry) * secs.size() + 63) / 64 * 64;
    for (size_t i = 0; i < secs.size(); ++i) {
        const uint64_t bytes = secs[i].count * secs[i].elem;
        tab[i] = Entry{secs[i].tag, secs[i].elem, secs[i].count, off, checksum(secs[i].data, bytes)};
        off = (off + bytes + 63) / 64 * 64;
    }
    hd.table_sum = checksum(tab.data(), sizeof(Entry) * tab.size());
    hd.header_sum = 0;
    hd.header_sum = checksum(&hd, sizeof(hd));
    const std::string tmp = std::string(path) + ".tmp." + std::to_string((long)getpid());
    {
        File fo;
        fo.f = std::fopen(tmp.c_str(), "wb");
        QMB_REQUIRE(fo.f, QMB_ERR_IO, std::string("cannot open ") + tmp + " for writing");
        auto put = [&](const void* p, size_t n) {
            if (n && std::fwrite(p, 1, n, fo.f) != n) {
                std::remove(tmp.c_str());
                throw Error{QMB_ERR_IO, std::string("write failed: ") + tmp};
            }
        };
        static const unsigned char zeros[64] = {0};
        uint64_t pos = 0;
        put(&hd, sizeof(hd));
        put(tab.data(), sizeof(Entry) * tab.size());
        pos = sizeof(hd) + sizeof(Entry) * tab.size();
        for (size_t i = 0; i < secs.size(); ++i) {
            put(zeros, tab[i].offset - pos);
            const uint64_t bytes = secs[i].count * secs[i].elem;
            put(secs[i].data, bytes);
            pos = tab[i].offset + bytes;
        }
        if (std::fflush(fo.f) != 0 || std::fclose(fo.f) != 0) {
            fo.f = nullptr;
            std::remove(tmp.c_str());
            throw Error{QMB_ERR_IO, std::string("write failed: ") + tmp};
        }
        fo.f = nullptr;
    }
    if (std::rename(tmp.c_str(), path) != 0) {
        std::remove(tmp.c_str());
        throw Error{QMB_ERR_IO, std::string("cannot rename ") + tmp + " to " + path};
    }
}

// A file read whole: header, table and payload checks done.
struct Loaded {
    Header hd{};
    std::vector<Entry> tab;
    std::vector<unsigned char> bytes;
    const Entry* find(uint32_t tag) const {
        for (const Entry& e : tab)
            if (e.tag == tag) return &e;
        return nullptr;
    }
    // payload of tag with the expected element size and count (count 0: any)
    const void* get(uint32_t tag, uint32_t elem, uint64_t count, uint64_t* n_out = nullptr) const {
        const Entry* e = find(tag);
        QMB_REQUIRE(e, QMB_ERR_CORRUPT, "table file lacks section " + std::to_string(tag));
        QMB_REQUIRE(e->elem_bytes == elem && (count == 0 || e->count == count), QMB_ERR_CORRUPT,
                    "table file section " + std::to_string(tag) + " has the wrong shape");
        if (n_out) *n_out = e->count;
        return bytes.data() + e->offset;
    }
};

Loaded read_file(const char* path, uint32_t kind) {
    QMB_REQUIRE(path && *path, QMB_ERR_INVALID, "empty path");
    File fi;
    fi.f = std::fopen(path, "rb");
    QMB_REQUIRE(fi.f, QMB_ERR_IO, std::string("cannot open ") + path);
    QMB_REQUIRE(std::fseek(fi.f, 0, SEEK_END) == 0, QMB_ERR_IO, std::string("cannot seek in ") + path);
    const long end = std::ftell(fi.f);
    QMB_REQUIRE(end >= 0, QMB_ERR_IO, std::string("cannot size ") + path);
    std::rewind(fi.f);
    Loaded L;
    L.bytes.resize((size_t)end);
    QMB_REQUIRE(std::fread(L.bytes.data(), 1, L.bytes.size(), fi.f) == L.bytes.size(), QMB_ERR_IO,
                std::string("read failed: ") + path);
    QMB_REQUIRE(L.bytes.size() >= sizeof(Header), QMB_ERR_CORRUPT, std::string(path) + ": shorter than a header");
    std::memcpy(&L.hd, L.bytes.data(), sizeof(Header));
    QMB_REQUIRE(std::memcmp(L.hd.magic, kMagic, 8) == 0, QMB_ERR_CORRUPT, std::string(path) + ": not a table file");
    QMB_REQUIRE(L.hd.byte_order == kByteOrder, QMB_ERR_UNSUPPORTED,
                std::string(path) + ": written with another byte order");
    Header h0 = L.hd;
    h0.header_sum = 0;
    QMB_REQUIRE(checksum(&h0, sizeof(h0)) == L.hd.header_sum, QMB_ERR_CORRUPT,
                std::string(path) + ": header checksum mismatch");
    QMB_REQUIRE(L.hd.version == kVersion, QMB_ERR_UNSUPPORTED,
                std::string(path) + ": format version " + std::to_string(L.hd.version) + ", this build reads " +
                    std::to_string(kVersion));
    QMB_REQUIRE(L.hd.kind == kind, QMB_ERR_INVALID,
                std::string(path) + ": holds table kind " + std::to_string(L.hd.kind) + ", expected " +
                    std::to_string(kind));
    const uint64_t n = L.hd.n_sections;
    QMB_REQUIRE(n <= 64 && sizeof(Header) + n * sizeof(Entry) <= L.bytes.size(), QMB_ERR_CORRUPT,
                std::string(path) + ": section table out of range");
    L.tab.resize(n);
    std::memcpy(L.tab.data(), L.bytes.data() + sizeof(Header), n * sizeof(Entry));
    QMB_REQUIRE(checksum(L.tab.data(), n * sizeof(Entry)) == L.hd.table_sum, QMB_ERR_CORRUPT,
                std::string(path) + ": section table checksum mismatch");
    for (const Entry& e : L.tab) {
        QMB_REQUIRE(e.elem_bytes >= 1 && e.elem_bytes <= 16 && e.count <= (uint64_t)1 << 40, QMB_ERR_CORRUPT,
                    std::string(path) + ": section shape out of range");
        const uint64_t bytes = e.count * e.elem_bytes;
        QMB_REQUIRE(e.offset <= L.bytes.size() && bytes <= L.bytes.size() - e.offset, QMB_ERR_CORRUPT,
                    std::string(path) + ": section runs past the end of the file (truncated?)");
        QMB_REQUIRE(checksum(L.bytes.data() + e.offset, bytes) == e.sum, QMB_ERR_CORRUPT,
                    std::string(path) + ": checksum mismatch in section " + std::to_string(e.tag));
    }
    return L;
}

uint64_t reps_checksum(qmb_sector_s* s) {
    if (!s->reps_sum) {
        std::vector<uint64_t> r(s->R);
        QMB_CUDA_TRY(cudaMemcpy(r.data(), s->reps.p, sizeof(uint64_t) * s->R, cudaMemcpyDeviceToHost));
        s->reps_sum = checksum(r.data(), sizeof(uint64_t) * r.size()) | 1;
    }
    return s->reps_sum;
}

uint64_t chars_checksum(const qmb_sector_s* s) {
    std::vector<double> c(2 * s->chars.size());
    for (size_t e = 0; e < s->chars.size(); ++e) {
        c[2 * e] = s->chars[e].real();
        c[2 * e + 1] = s->chars[e].imag();
    }
    return checksum(c.data(), sizeof(double) * c.size());
}

// Sector identity recorded in a matrix file: meta[16..26].
void sector_fingerprint(qmb_sector_s* s, uint64_t* m) {
    m[0] = (uint64_t)s->L;
    m[1] = (uint64_t)s->n_up;
    m[2] = (uint64_t)s->G;
    m[3] = (uint64_t)s->flip;
    m[4] = (uint64_t)s->R;
    m[5] = checksum(s->perm.data(), sizeof(uint32_t) * s->perm.size());
    m[6] = reps_checksum(s);
    m[7] = chars_checksum(s);
    m[8] = dbits(s->tol_norm);
    m[9] = (uint64_t)s->n_active;
    m[10] = 0;
}

template <class T>
std::vector<T> download(const DevBuf<T>& b, size_t count) {
    std::vector<T> h(count);
    if (count) QMB_CUDA_TRY(cudaMemcpy(h.data(), b.p, sizeof(T) * count, cudaMemcpyDeviceToHost));
    return h;
}

template <class T>
void upload(DevBuf<T>& b, const void* src, size_t count) {
    b.alloc(std::max<size_t>(count, 1));
    if (count) QMB_CUDA_TRY(cudaMemcpy(b.p, src, sizeof(T) * count, cudaMemcpyHostToDevice));
}

}  // namespace
}  // namespace qmb

using namespace qmb;

extern "C" qmb_status qmb_sector_save(qmb_sector s, const char* path) {
    return guarded([&] {
        QMB_REQUIRE(s && path, QMB_ERR_INVALID, "null argument");
        DeviceGuard dg(s->device);
        std::vector<uint64_t> reps = download(s->reps, (size_t)s->R);
        std::vector<double> ch(2 * s->chars.size());
        for (size_t e = 0; e < s->chars.size(); ++e) {
            ch[2 * e] = s->chars[e].real();
            ch[2 * e + 1] = s->chars[e].imag();
        }
        uint64_t meta[27] = {};
        meta[0] = (uint64_t)s->L;
        meta[1] = (uint64_t)s->n_up;
        meta[2] = (uint64_t)s->G;
        meta[3] = (uint64_t)s->flip;
        meta[4] = (uint64_t)s->R;
        meta[5] = s->has_irrep ? 1 : 0;
        meta[6] = s->has_irrep ? (uint64_t)s->n_active : 0;
        meta[7] = dbits(s->tol_norm);
        meta[8] = (uint64_t)s->n_ext;
        std::vector<Section> secs = {{TAG_PERM, 4, (uint64_t)s->perm.size(), s->perm.data()},
                                     {TAG_REPS, 8, (uint64_t)reps.size(), reps.data()}};
        if (s->has_irrep) secs.push_back({TAG_CHARS, 16, (uint64_t)s->chars.size(), ch.data()});
        write_file(path, KIND_SECTOR, meta, secs);
    });
}

extern "C" qmb_status qmb_sector_load(const char* path, int device, qmb_sector* out) {
    return guarded([&] {
        QMB_REQUIRE(path && out, QMB_ERR_INVALID, "null argument");
        *out = nullptr;
        Loaded F = read_file(path, KIND_SECTOR);
        const uint64_t* m = F.hd.meta;
        QMB_REQUIRE(m[0] >= 1 && m[0] <= 64 && m[1] <= m[0] && m[2] >= 1 && m[2] <= (uint64_t)kMaxPerm && m[3] <= 1,
                    QMB_ERR_CORRUPT, std::string(path) + ": sector parameters out of range");
        const int L = (int)m[0], G = (int)m[2];
        const uint32_t* perm = (const uint32_t*)F.get(TAG_PERM, 4, (uint64_t)G * L);
        const uint64_t* reps = (const uint64_t*)F.get(TAG_REPS, 8, m[4]);
        qmb_sector_desc d;
        d.L = L;
        d.n_up = (int)m[1];
        d.n_perm = G;
        d.perm = perm;
        d.spin_flip = (int)m[3];
        d.device = device;
        std::unique_ptr<qmb_sector_s> s(sector_from_reps(&d, reps, (int64_t)m[4]));
        DeviceGuard dg(device);
        if (m[5]) {
            const double* ch = (const double*)F.get(TAG_CHARS, 16, (uint64_t)s->n_ext);
            sector_select_irrep(s.get(), ch, bitsd(m[7]));
            QMB_REQUIRE((uint64_t)s->n_active == m[6], QMB_ERR_CORRUPT,
                        std::string(path) + ": the irrep's active rows differ from the file's count");
        }
        *out = s.release();
    });
}

extern "C" qmb_status qmb_ham_save(qmb_ham h, const char* path) {
    return guarded([&] {
        QMB_REQUIRE(h && path, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(h->irrep_gen == h->sector->irrep_gen, QMB_ERR_INVALID,
                    "the sector's irrep changed since the handle was built");
        DeviceGuard dg(h->device);
        const size_t es = h->cplx ? 16 : 8, es32 = h->cplx ? 8 : 4;
        const size_t pad = (size_t)std::max<int64_t>(h->padded, 1), n = (size_t)h->n;
        auto off = download(h->slice_off, (size_t)h->n_slices + 1);
        auto wid = download(h->slice_w, (size_t)h->n_slices);
        auto col = download(h->col, pad);
        std::vector<unsigned char> v64, v32, d64, d32;
        if (h->val64.p) v64 = download(h->val64, pad * es);
        if (h->val32.p) v32 = download(h->val32, pad * es32);
        d64 = download(h->diag64, n * es);
        if (h->diag32.p) d32 = download(h->diag32, n * es32);
        auto tn = download(h->t_nops, (size_t)h->n_terms);
        auto to = download(h->t_ops, (size_t)h->n_terms * h->n_col);
        auto ts = download(h->t_scalar, (size_t)h->n_terms);
        uint64_t meta[27] = {};
        meta[0] = (uint64_t)h->n;
        meta[1] = h->cplx ? 1 : 0;
        meta[2] = (uint64_t)h->prec;
        meta[3] = (uint64_t)h->n_slices;
        meta[4] = (uint64_t)h->padded;
        meta[5] = (uint64_t)h->nnz;
        meta[6] = (uint64_t)h->max_row;
        meta[7] = (uint64_t)h->n_terms;
        meta[8] = (uint64_t)h->n_col;
        sector_fingerprint(h->sector, meta + 16);
        std::vector<Section> secs = {{TAG_SLICE_OFF, 8, off.size(), off.data()},
                                     {TAG_SLICE_W, 4, wid.size(), wid.data()},
                                     {TAG_COL, 4, col.size(), col.data()},
                                     {TAG_DIAG64, (uint32_t)es, n, d64.data()},
                                     {TAG_T_NOPS, 4, tn.size(), tn.data()},
                                     {TAG_T_OPS, 2, to.size(), to.data()},
                                     {TAG_T_SCALAR, 16, ts.size(), ts.data()}};
        if (!v64.empty()) secs.push_back({TAG_VAL64, (uint32_t)es, pad, v64.data()});
        if (!v32.empty()) secs.push_back({TAG_VAL32, (uint32_t)es32, pad, v32.data()});
        if (!d32.empty()) secs.push_back({TAG_DIAG32, (uint32_t)es32, n, d32.data()});
        write_file(path, KIND_HAM, meta, secs);
    });
}

extern "C" qmb_status qmb_ham_load(qmb_sector s, const char* path, qmb_ham* out) {
    return guarded([&] {
        QMB_REQUIRE(s && path && out, QMB_ERR_INVALID, "null argument");
        *out = nullptr;
        QMB_REQUIRE(s->has_irrep, QMB_ERR_INVALID, "select the sector's irrep before loading a matrix");
        DeviceGuard dg(s->device);
        Loaded F = read_file(path, KIND_HAM);
        const uint64_t* m = F.hd.meta;
        uint64_t fp[11];
        sector_fingerprint(s, fp);
        static const char* what[11] = {"L", "n_up", "group size", "spin inversion", "orbit count",
                                       "group elements", "representatives", "irrep characters",
                                       "norm tolerance", "active rows", "reserved"};
        for (int i = 0; i < 11; ++i)
            QMB_REQUIRE(m[16 + i] == fp[i], QMB_ERR_INVALID,
                        std::string(path) + ": written for another sector or irrep (" + what[i] + " differ)");
        QMB_REQUIRE(m[0] == (uint64_t)s->n_active && m[1] <= 1 && m[7] <= (uint64_t)kMaxTerms && m[8] >= 1 &&
                        m[8] <= (uint64_t)kMaxCol && m[3] == (m[0] + 31) / 32,
                    QMB_ERR_CORRUPT, std::string(path) + ": matrix parameters out of range");
        auto h = std::make_unique<qmb_ham_s>();
        h->sector = s;
        h->device = s->device;
        h->irrep_gen = s->irrep_gen;
        h->n = (int64_t)m[0];
        h->cplx = m[1] != 0;
        h->prec = (int)m[2];
        h->n_slices = (int64_t)m[3];
        h->padded = (int64_t)m[4];
        h->nnz = (int64_t)m[5];
        h->max_row = (int)m[6];
        h->n_terms = (int)m[7];
        h->n_col = (int)m[8];
        const size_t es = h->cplx ? 16 : 8, es32 = h->cplx ? 8 : 4;
        const uint64_t pad = (uint64_t)std::max<int64_t>(h->padded, 1), n = (uint64_t)h->n;
        const int64_t* off = (const int64_t*)F.get(TAG_SLICE_OFF, 8, (uint64_t)h->n_slices + 1);
        QMB_REQUIRE(off[h->n_slices] == h->padded, QMB_ERR_CORRUPT, std::string(path) + ": slice offsets inconsistent");
        const int* wid = (const int*)F.get(TAG_SLICE_W, 4, (uint64_t)h->n_slices);
        for (int64_t i = 0; i < h->n_slices; ++i)
            QMB_REQUIRE(wid[i] >= 0 && off[i] >= 0 && (uint64_t)off[i] + 32ull * (uint64_t)wid[i] <= pad,
                        QMB_ERR_CORRUPT, std::string(path) + ": slice outside the stored entries");
        const uint32_t* col = (const uint32_t*)F.get(TAG_COL, 4, pad);
        for (uint64_t i = 0; i < pad; ++i)
            QMB_REQUIRE(col[i] < n, QMB_ERR_CORRUPT, std::string(path) + ": column index out of range");
        upload<int64_t>(h->slice_off, off, (size_t)h->n_slices + 1);
        upload<int>(h->slice_w, wid, (size_t)h->n_slices);
        upload<uint32_t>(h->col, col, pad);
        upload<unsigned char>(h->diag64, F.get(TAG_DIAG64, (uint32_t)es, n), n * es);
        if (F.find(TAG_VAL64)) upload<unsigned char>(h->val64, F.get(TAG_VAL64, (uint32_t)es, pad), pad * es);
        if (F.find(TAG_VAL32)) upload<unsigned char>(h->val32, F.get(TAG_VAL32, (uint32_t)es32, pad), pad * es32);
        if (F.find(TAG_DIAG32)) upload<unsigned char>(h->diag32, F.get(TAG_DIAG32, (uint32_t)es32, n), n * es32);
        QMB_REQUIRE(((h->prec & QMB_PREC_FP64) == 0 || h->val64.p) && ((h->prec & QMB_PREC_FP32) == 0 || h->val32.p),
                    QMB_ERR_CORRUPT, std::string(path) + ": stored values do not match the precision mask");
        const int* tn = (const int*)F.get(TAG_T_NOPS, 4, (uint64_t)h->n_terms);
        const uint16_t* to = (const uint16_t*)F.get(TAG_T_OPS, 2, (uint64_t)h->n_terms * h->n_col);
        for (int i = 0; i < h->n_terms; ++i) {
            QMB_REQUIRE(tn[i] >= 0 && tn[i] <= h->n_col, QMB_ERR_CORRUPT, std::string(path) + ": term table out of range");
            for (int j = 0; j < tn[i]; ++j)
                QMB_REQUIRE((to[(size_t)i * h->n_col + j] & 0xff) < s->L, QMB_ERR_CORRUPT,
                            std::string(path) + ": term site out of range");
        }
        upload<int>(h->t_nops, tn, (size_t)h->n_terms);
        upload<uint16_t>(h->t_ops, to, (size_t)h->n_terms * h->n_col);
        const double2* tsc = (const double2*)F.get(TAG_T_SCALAR, 16, (uint64_t)h->n_terms);
        upload<double2>(h->t_scalar, tsc, (size_t)h->n_terms);
        {
            // the hop form, as qmb_ham_create derives it from the same table
            std::vector<int> codes((size_t)h->n_terms * h->n_col), sites(codes.size());
            std::vector<double> sc(2 * (size_t)h->n_terms);
            for (size_t i = 0; i < codes.size(); ++i) {
                codes[i] = to[i] >> 8;
                sites[i] = to[i] & 0xff;
            }
            for (int i = 0; i < h->n_terms; ++i) {
                sc[2 * (size_t)i] = tsc[i].x;
                sc[2 * (size_t)i + 1] = tsc[i].y;
            }
            qmb_terms t{};
            t.n_terms = h->n_terms;
            t.n_col = h->n_col;
            t.n_ops = tn;
            t.op_code = codes.data();
            t.op_site = sites.data();
            t.scalar = sc.data();
            hop_form(h.get(), &t);
        }
        h->err.alloc(1);
        h->err.zero();
        QMB_CUDA_TRY(cudaDeviceSynchronize());
        build_cb(h.get());  // the coded FP32 layout, as qmb_ham_create builds it
        *out = h.release();
    });
}

extern "C" qmb_status qmb_ref_ell_save(const char* path, int64_t n_rows, int width, const uint32_t* ind,
                                       const void* val, const int16_t* track, int is_complex) {
    return guarded([&] {
        QMB_REQUIRE(path && ind && val && track, QMB_ERR_INVALID, "null argument");
        QMB_REQUIRE(n_rows >= 1 && width >= 1, QMB_ERR_INVALID, "bad sizes");
        const uint64_t nw = (uint64_t)n_rows * (uint64_t)width;
        uint64_t meta[27] = {};
        meta[0] = (uint64_t)n_rows;
        meta[1] = (uint64_t)width;
        meta[2] = is_complex ? 1 : 0;
        std::vector<Section> secs = {{TAG_IND, 4, nw, ind},
                                     {TAG_VAL, is_complex ? 8u : 4u, nw, val},
                                     {TAG_TRACK, 2, (uint64_t)n_rows, track}};
        write_file(path, KIND_REF_ELL, meta, secs);
    });
}

extern "C" qmb_status qmb_ref_ell_load(const char* path, int64_t* n_rows, int* width, int* is_complex,
                                       uint32_t* ind, void* val, int16_t* track, int64_t cap_rows) {
    return guarded([&] {
        QMB_REQUIRE(path && n_rows && width && is_complex, QMB_ERR_INVALID, "null argument");
        Loaded F = read_file(path, KIND_REF_ELL);
        const uint64_t* m = F.hd.meta;
        QMB_REQUIRE(m[0] >= 1 && m[1] >= 1 && m[1] < (1u << 16) && m[2] <= 1, QMB_ERR_CORRUPT,
                    std::string(path) + ": table parameters out of range");
        *n_rows = (int64_t)m[0];
        *width = (int)m[1];
        *is_complex = (int)m[2];
        if (!ind && !val && !track) return;  // size query
        QMB_REQUIRE(ind && val && track, QMB_ERR_INVALID, "give all three buffers or none");
        QMB_REQUIRE(cap_rows >= (int64_t)m[0], QMB_ERR_INVALID, "buffers hold fewer rows than the file");
        const uint64_t nw = m[0] * m[1];
        const uint32_t es = m[2] ? 8u : 4u;
        std::memcpy(ind, F.get(TAG_IND, 4, nw), 4 * nw);
        std::memcpy(val, F.get(TAG_VAL, es, nw), (size_t)es * nw);
        std::memcpy(track, F.get(TAG_TRACK, 2, m[0]), 2 * m[0]);
    });
}
