// Database file: a length-aware, multi-volume on-disk form of the subject
// database, and its staged upload into HBM.
//
// The reference builds a ".gpu" file of 4-byte-interleaved, group-padded
// subjects capped at 4 GB per volume (functions.cpp:364-613, the cap at
// :481-485) and reads it whole into host memory before one synchronous copy
// (functions.cpp:620-699).  Here a file holds:
//
//   header (64 B)   magic "BPDB0001", flags (bit 0: subjects sorted by
//                   length, longest first), subject and residue counts,
//                   volume count, volume residue cap
//   volume table    per volume: first subject, subject count, residue count,
//                   file offsets of its residues and of its offsets
//   oid map         int32 original index of every stored subject (sorted files)
//   volumes         residues (uint8, each volume 4 KiB aligned) and int64
//                   offsets relative to the volume's first residue
//
// bp_db_open maps the file and streams each volume through two pinned
// staging buffers (host copy of one overlapping the DMA of the other) into
// one flat device residue array and one offsets array -- the layout every
// search uses -- then checks the residue codes on the device.
#include <fcntl.h>
#include <stdio.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

#include "bp_internal.h"

namespace {

constexpr char kMagic[8] = {'B', 'P', 'D', 'B', '0', '0', '0', '1'};
constexpr int64_t kAlign = 4096;
constexpr size_t kStage = (size_t)64 << 20;     // bytes per pinned staging buffer

struct FileHeader {
    char magic[8];
    uint32_t flags;
    uint32_t n_volumes;
    int64_t n_subjects;
    int64_t n_residues;
    int64_t volume_residues;
    int64_t reserved[3];
};
static_assert(sizeof(FileHeader) == 64, "header layout");

struct VolumeEntry {
    int64_t first_subject, n_subjects, n_residues;
    int64_t residues_at, offsets_at;     // file offsets
    int64_t reserved;
};
static_assert(sizeof(VolumeEntry) == 48, "volume entry layout");

int64_t align_up(int64_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// Copies n bytes with up to `threads` host threads (page-cache reads into
// pinned memory are bound by one core's copy rate otherwise).
void parallel_copy(uint8_t* dst, const uint8_t* src, size_t n, int threads) {
    const size_t per = (n + (size_t)threads - 1) / (size_t)threads;
    if (threads <= 1 || n < ((size_t)4 << 20)) {
        memcpy(dst, src, n);
        return;
    }
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; ++t) {
        const size_t lo = (size_t)t * per, hi = std::min(n, lo + per);
        if (lo >= hi) break;
        ts.emplace_back([=] { memcpy(dst + lo, src + lo, hi - lo); });
    }
    for (auto& t : ts) t.join();
}

bool write_all(FILE* f, const void* p, size_t n) { return n == 0 || fwrite(p, 1, n, f) == n; }

bool pad_to(FILE* f, int64_t at) {
    const long cur = ftell(f);
    if (cur < 0 || cur > at) return false;
    static const char zeros[4096] = {0};
    for (int64_t left = at - cur; left > 0;) {
        const size_t k = (size_t)std::min<int64_t>(left, sizeof(zeros));
        if (!write_all(f, zeros, k)) return false;
        left -= (int64_t)k;
    }
    return true;
}

// A mapped, validated file.
struct Mapped {
    const uint8_t* base = nullptr;
    size_t size = 0;
    FileHeader h{};
    const VolumeEntry* vols = nullptr;
    const int32_t* oids = nullptr;
    std::string err;

    ~Mapped() {
        if (base) munmap((void*)base, size);
    }

    bool open(const char* path) {
        const int fd = ::open(path, O_RDONLY);
        if (fd < 0) {
            err = std::string("cannot open ") + path;
            return false;
        }
        struct stat st;
        if (fstat(fd, &st) != 0 || st.st_size < (off_t)sizeof(FileHeader)) {
            ::close(fd);
            err = "not a database file (too short)";
            return false;
        }
        size = (size_t)st.st_size;
        void* p = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
        ::close(fd);
        if (p == MAP_FAILED) {
            err = "mmap failed";
            return false;
        }
        base = (const uint8_t*)p;
        memcpy(&h, base, sizeof(h));
        if (memcmp(h.magic, kMagic, 8) != 0) return fail("bad magic");
        if (h.n_subjects < 0 || h.n_subjects >= (1LL << 31) || h.n_residues < 0 || h.n_volumes > (1u << 20))
            return fail("bad counts");
        const size_t vt = sizeof(FileHeader) + (size_t)h.n_volumes * sizeof(VolumeEntry);
        const size_t om = (h.flags & 1) ? (size_t)h.n_subjects * 4 : 0;
        if (vt + om > size) return fail("truncated tables");
        vols = (const VolumeEntry*)(base + sizeof(FileHeader));
        oids = (h.flags & 1) ? (const int32_t*)(base + vt) : nullptr;
        int64_t s = 0, r = 0;
        for (uint32_t v = 0; v < h.n_volumes; ++v) {
            const VolumeEntry& e = vols[v];
            if (e.first_subject != s || e.n_subjects < 0 || e.n_residues < 0) return fail("bad volume table");
            if (e.residues_at < 0 || e.residues_at + e.n_residues > (int64_t)size ||
                e.offsets_at < 0 || e.offsets_at + (e.n_subjects + 1) * 8 > (int64_t)size || (e.offsets_at & 7))
                return fail("volume beyond the end of the file");
            const int64_t* off = (const int64_t*)(base + e.offsets_at);
            if (off[0] != 0 || off[e.n_subjects] != e.n_residues) return fail("bad volume offsets");
            s += e.n_subjects;
            r += e.n_residues;
        }
        if (s != h.n_subjects || r != h.n_residues) return fail("volume totals differ from the header");
        return true;
    }

    bool fail(const char* why) {
        err = std::string("database file: ") + why;
        return false;
    }
};

}  // namespace

extern "C" {

bp_status bp_dbfile_write(const char* path, const uint8_t* residues, int64_t n_residues, const int64_t* offsets,
                          int32_t n_subjects, int64_t volume_residues, int32_t sort_by_length) {
    if (!path || !offsets || n_subjects < 0 || n_residues < 0 || (n_residues > 0 && !residues))
        return BP_ERR_INVALID;
    if (offsets[0] != 0 || offsets[n_subjects] != n_residues) return BP_ERR_INVALID;
    for (int32_t i = 0; i < n_subjects; ++i)
        if (offsets[i + 1] < offsets[i] || offsets[i + 1] - offsets[i] > (1 << 29)) return BP_ERR_INVALID;
    for (int64_t i = 0; i < n_residues; ++i)
        if (residues[i] >= BP_ALPHABET) return BP_ERR_INVALID;
    if (volume_residues <= 0) volume_residues = (int64_t)1 << 30;
    // stored order: longest first when sorting (stable, so ties keep their order)
    std::vector<int32_t> order(n_subjects);
    std::iota(order.begin(), order.end(), 0);
    if (sort_by_length)
        std::stable_sort(order.begin(), order.end(), [&](int32_t a, int32_t b) {
            return offsets[a + 1] - offsets[a] > offsets[b + 1] - offsets[b];
        });
    // volumes: consecutive stored subjects up to volume_residues (at least one subject)
    std::vector<VolumeEntry> vols;
    for (int32_t s = 0; s < n_subjects;) {
        VolumeEntry v{};
        v.first_subject = s;
        while (s < n_subjects) {
            const int64_t len = offsets[order[s] + 1] - offsets[order[s]];
            if (v.n_subjects > 0 && v.n_residues + len > volume_residues) break;
            v.n_residues += len;
            v.n_subjects += 1;
            ++s;
        }
        vols.push_back(v);
    }
    FileHeader h{};
    memcpy(h.magic, kMagic, 8);
    h.flags = sort_by_length ? 1u : 0u;
    h.n_volumes = (uint32_t)vols.size();
    h.n_subjects = n_subjects;
    h.n_residues = n_residues;
    h.volume_residues = volume_residues;
    int64_t at = align_up((int64_t)sizeof(FileHeader) + (int64_t)vols.size() * (int64_t)sizeof(VolumeEntry) +
                          (sort_by_length ? (int64_t)n_subjects * 4 : 0));
    for (VolumeEntry& v : vols) {
        v.residues_at = at;
        at = align_up(at + v.n_residues);
        v.offsets_at = at;
        at = align_up(at + (v.n_subjects + 1) * 8);
    }
    FILE* f = fopen(path, "wb");
    if (!f) return BP_ERR_INVALID;
    bool ok = write_all(f, &h, sizeof(h)) && write_all(f, vols.data(), vols.size() * sizeof(VolumeEntry));
    if (ok && sort_by_length) ok = write_all(f, order.data(), order.size() * 4);
    std::vector<int64_t> voff;
    for (const VolumeEntry& v : vols) {
        if (!ok) break;
        ok = pad_to(f, v.residues_at);
        for (int64_t k = 0; ok && k < v.n_subjects; ++k) {
            const int32_t o = order[(size_t)(v.first_subject + k)];
            ok = write_all(f, residues + offsets[o], (size_t)(offsets[o + 1] - offsets[o]));
        }
        voff.assign((size_t)v.n_subjects + 1, 0);
        for (int64_t k = 0; k < v.n_subjects; ++k) {
            const int32_t o = order[(size_t)(v.first_subject + k)];
            voff[(size_t)k + 1] = voff[(size_t)k] + (offsets[o + 1] - offsets[o]);
        }
        if (ok) ok = pad_to(f, v.offsets_at) && write_all(f, voff.data(), voff.size() * 8);
    }
    if (ok) ok = pad_to(f, at);
    if (fclose(f) != 0) ok = false;
    return ok ? BP_OK : BP_ERR_INVALID;
}

bp_status bp_dbfile_info(const char* path, int32_t* n_subjects, int64_t* n_residues, int32_t* n_volumes,
                         int32_t* sorted) {
    Mapped m;
    if (!path || !m.open(path)) return BP_ERR_INVALID;
    if (n_subjects) *n_subjects = (int32_t)m.h.n_subjects;
    if (n_residues) *n_residues = m.h.n_residues;
    if (n_volumes) *n_volumes = (int32_t)m.h.n_volumes;
    if (sorted) *sorted = (int32_t)(m.h.flags & 1);
    return BP_OK;
}

bp_status bp_dbfile_read_host(const char* path, uint8_t* residues, int64_t* offsets, int32_t* oids) {
    Mapped m;
    if (!path || !m.open(path)) return BP_ERR_INVALID;
    int64_t r = 0;
    if (offsets) offsets[0] = 0;
    for (uint32_t v = 0; v < m.h.n_volumes; ++v) {
        const VolumeEntry& e = m.vols[v];
        const int64_t* off = (const int64_t*)(m.base + e.offsets_at);
        if (residues && e.n_residues) memcpy(residues + r, m.base + e.residues_at, (size_t)e.n_residues);
        if (offsets)
            for (int64_t k = 1; k <= e.n_subjects; ++k) offsets[e.first_subject + k] = r + off[k];
        r += e.n_residues;
    }
    if (oids)
        for (int64_t i = 0; i < m.h.n_subjects; ++i) oids[i] = m.oids ? m.oids[i] : (int32_t)i;
    return BP_OK;
}

bp_status bp_db_open(bp_engine* e, const char* path, bp_db** out) {
    if (!e || !path || !out) return bp_set_error(e, BP_ERR_INVALID, "bp_db_open: bad argument");
    *out = nullptr;
    Mapped m;
    if (!m.open(path)) return bp_set_error(e, BP_ERR_INVALID, m.err);
    if (cudaSetDevice(e->device) != cudaSuccess) return bp_set_cuda_error(e, cudaGetLastError(), "cudaSetDevice");
    bp_db* db = nullptr;
    bp_status st = bp_db_alloc(e, m.h.n_residues, (int32_t)m.h.n_subjects, &db);
    if (st != BP_OK) return st;
    // global offsets on the host (chunk planning needs them too), checked as
    // they are assembled
    db->h_off.assign((size_t)m.h.n_subjects + 1, 0);
    int64_t r = 0;
    for (uint32_t v = 0; v < m.h.n_volumes; ++v) {
        const VolumeEntry& ve = m.vols[v];
        const int64_t* off = (const int64_t*)(m.base + ve.offsets_at);
        for (int64_t k = 1; k <= ve.n_subjects; ++k) {
            if (off[k] < off[k - 1] || off[k] - off[k - 1] > (1 << 29)) {
                bp_db_destroy(db);
                return bp_set_error(e, BP_ERR_INVALID, "database file: offsets must be non-decreasing");
            }
            db->h_off[(size_t)(ve.first_subject + k)] = r + off[k];
        }
        r += ve.n_residues;
    }
    // residues: two pinned staging buffers, host copy of one while the other's DMA runs
    uint8_t* stage[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    cudaError_t err = cudaSuccess;
    for (int i = 0; i < 2 && err == cudaSuccess; ++i) {
        err = cudaMallocHost((void**)&stage[i], kStage);
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming);
    }
    int slot = 0;
    int64_t dst = 0;
    const int copy_threads = (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    for (uint32_t v = 0; v < m.h.n_volumes && err == cudaSuccess; ++v) {
        const VolumeEntry& ve = m.vols[v];
        for (int64_t k = 0; k < ve.n_residues && err == cudaSuccess; k += (int64_t)kStage) {
            const size_t n = (size_t)std::min<int64_t>((int64_t)kStage, ve.n_residues - k);
            err = cudaEventSynchronize(done[slot]);        // the buffer's previous DMA is finished
            if (err != cudaSuccess) break;
            parallel_copy(stage[slot], m.base + ve.residues_at + k, n, copy_threads);
            err = cudaMemcpyAsync(db->d_res + dst, stage[slot], n, cudaMemcpyHostToDevice, e->stream);
            if (err == cudaSuccess) err = cudaEventRecord(done[slot], e->stream);
            dst += (int64_t)n;
            slot ^= 1;
        }
    }
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(db->d_off, db->h_off.data(), db->h_off.size() * 8, cudaMemcpyHostToDevice, e->stream);
    if (err == cudaSuccess) err = cudaStreamSynchronize(e->stream);
    for (int i = 0; i < 2; ++i) {
        if (done[i]) cudaEventDestroy(done[i]);
        if (stage[i]) cudaFreeHost(stage[i]);
    }
    if (err != cudaSuccess) {
        bp_db_destroy(db);
        return bp_set_cuda_error(e, err, "bp_db_open: upload");
    }
    st = bp_db_finish(e, db);
    if (st != BP_OK) {
        bp_db_destroy(db);
        return st;
    }
    *out = db;
    return BP_OK;
}

}  // extern "C"
