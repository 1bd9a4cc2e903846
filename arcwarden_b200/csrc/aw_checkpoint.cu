// aw_checkpoint.cu — checkpoint and restart in the reference's file format
// (include/pic/checkpoint.hpp:1-17: header, deck block, git block, manifest,
// then the array payloads in manifest order, which the reference leaves for a
// later milestone and this library writes).
//
// Layout (little-endian): u32 magic "ARCW", u32 version 1, u64 rng_seed,
// i64 step, f64 time, f64 S_d, f64 eps_L; u64 n + deck text; u64 n + git hash;
// u32 narrays, per array u32 name_len + name, u32 dtype (0 f32, 1 f64, 2 i32,
// 3 u64), u64 count; the payloads.
//
// Arrays: the particle SoA x y ux uy uz w (f32) and cell (i32, when bound);
// acc_src, the pending fixed-point deposit of the current state (u64,
// nsrc x ncell); devstate, the library's device state block (u64 words: deposit
// scales, |u| maxima, rms, step); the bound caller fields (f32). A restart reads
// all of them back, so the run continues bit for bit.
//
// Writing: the arrays are first copied device to device into a snapshot buffer
// on the context's stream (HBM speed), then a host thread streams the snapshot
// to the file through two pinned buffers on a stream of its own, while the run
// goes on. aw_checkpoint_wait joins it.
#include "aw_internal.h"

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace aw {

struct CkWriter {
    std::thread th;
    std::string err;
    void* snap = nullptr;            // device snapshot of the arrays
    size_t cap = 0, used = 0;        // its size, the bytes of the file being written
    void* pin[2] = {nullptr, nullptr};
    cudaStream_t s = nullptr;
    cudaEvent_t taken = nullptr, done[2] = {nullptr, nullptr};
};

namespace {

constexpr uint32_t kMagic = 0x57435241u;   // "ARCW"
constexpr uint32_t kVersion = 1;
constexpr size_t kChunkBytes = size_t(32) << 20;
enum : uint32_t { kF32 = 0, kF64 = 1, kI32 = 2, kU64 = 3 };
static_assert(sizeof(DevState) % 8 == 0, "devstate is stored as u64 words");

struct Arr {
    std::string name;
    uint32_t dtype;
    uint64_t count;
    void* dev;
    size_t bytes() const { return count * ((dtype == kF32 || dtype == kI32) ? 4 : 8); }
};

std::vector<Arr> arrays_of(const Ctx& c) {
    std::vector<Arr> v;
    const uint64_t n = static_cast<uint64_t>(c.parts.n), nc = static_cast<uint64_t>(c.geo.ncell);
    auto add = [&](const char* nm, uint32_t t, uint64_t cnt, void* p) {
        if (p && cnt) v.push_back({nm, t, cnt, p});
    };
    add("x", kF32, n, c.parts.x);
    add("y", kF32, n, c.parts.y);
    add("ux", kF32, n, c.parts.ux);
    add("uy", kF32, n, c.parts.uy);
    add("uz", kF32, n, c.parts.uz);
    add("w", kF32, n, c.parts.w);
    add("cell", kI32, n, c.parts.cell);
    add("acc_src", kU64, static_cast<uint64_t>(c.nsrc()) * nc, c.acc_src);
    add("devstate", kU64, sizeof(DevState) / 8, c.st);
    const std::pair<const char*, float*> f[] = {{"Ex", c.fld.Ex}, {"Ey", c.fld.Ey}, {"Ez", c.fld.Ez},
                                                {"Bx", c.fld.Bx}, {"By", c.fld.By}, {"Bz", c.fld.Bz}};
    for (const auto& e : f) add(e.first, kF32, nc, e.second);
    return v;
}

// The arrays a restart must find (the fields are optional).
bool required(const std::string& nm) { return nm != "Ex" && nm != "Ey" && nm != "Ez" && nm != "Bx" && nm != "By" && nm != "Bz"; }

struct File {
    std::FILE* f = nullptr;
    ~File() { if (f) std::fclose(f); }
    void put(const void* p, size_t n) {
        if (n && std::fwrite(p, 1, n, f) != n) throw Error(AW_ERR_STATE, "checkpoint: short write");
    }
    void get(void* p, size_t n) {
        if (n && std::fread(p, 1, n, f) != n) throw Error(AW_ERR_STATE, "checkpoint: short read (payload missing?)");
    }
    void put_str(const std::string& s) { const uint64_t n = s.size(); put(&n, 8); put(s.data(), s.size()); }
    std::string get_str() {
        uint64_t n = 0;
        get(&n, 8);
        need(n <= (uint64_t(1) << 30), AW_ERR_STATE, "checkpoint: string block too long");
        std::string s(n, '\0');
        get(&s[0], n);
        return s;
    }
};

struct Header {
    uint64_t seed = 0;
    int64_t step = 0;
    double time = 0.0, sd = 1.0, eps_l = 0.0;
    std::string deck, git;
    std::vector<Arr> manifest;      // dev unused
};

void write_header(File& f, const Header& h) {
    const uint32_t magic = kMagic, ver = kVersion;
    f.put(&magic, 4); f.put(&ver, 4);
    f.put(&h.seed, 8); f.put(&h.step, 8); f.put(&h.time, 8); f.put(&h.sd, 8); f.put(&h.eps_l, 8);
    f.put_str(h.deck);
    f.put_str(h.git);
    const uint32_t na = static_cast<uint32_t>(h.manifest.size());
    f.put(&na, 4);
    for (const Arr& a : h.manifest) {
        const uint32_t nl = static_cast<uint32_t>(a.name.size());
        f.put(&nl, 4); f.put(a.name.data(), nl); f.put(&a.dtype, 4); f.put(&a.count, 8);
    }
}

Header read_header(File& f) {
    Header h;
    uint32_t magic = 0, ver = 0;
    f.get(&magic, 4); f.get(&ver, 4);
    need(magic == kMagic, AW_ERR_STATE, "checkpoint: bad magic");
    need(ver <= kVersion, AW_ERR_STATE, "checkpoint: version newer than this reader");
    f.get(&h.seed, 8); f.get(&h.step, 8); f.get(&h.time, 8); f.get(&h.sd, 8); f.get(&h.eps_l, 8);
    h.deck = f.get_str();
    h.git = f.get_str();
    uint32_t na = 0;
    f.get(&na, 4);
    need(na <= 4096, AW_ERR_STATE, "checkpoint: manifest too long");
    for (uint32_t i = 0; i < na; ++i) {
        Arr a{};
        uint32_t nl = 0;
        f.get(&nl, 4);
        need(nl <= 256, AW_ERR_STATE, "checkpoint: array name too long");
        a.name.resize(nl);
        f.get(&a.name[0], nl);
        f.get(&a.dtype, 4);
        f.get(&a.count, 8);
        need(a.dtype <= kU64, AW_ERR_STATE, "checkpoint: bad dtype");
        h.manifest.push_back(a);
    }
    return h;
}

void writer_resources(CkWriter& w) {
    if (!w.s) {
        AW_CUDA(cudaStreamCreateWithFlags(&w.s, cudaStreamNonBlocking));
        AW_CUDA(cudaEventCreateWithFlags(&w.taken, cudaEventDisableTiming));
        for (int k = 0; k < 2; ++k) {
            AW_CUDA(cudaEventCreateWithFlags(&w.done[k], cudaEventDisableTiming));
            AW_CUDA(cudaMallocHost(&w.pin[k], kChunkBytes));
        }
    }
}

// Stream the device snapshot to the file (runs on the writer thread).
void stream_out(CkWriter& w, int device, const std::string& path, const Header& h) {
    try {
        AW_CUDA(cudaSetDevice(device));
        File f;
        f.f = std::fopen(path.c_str(), "wb");
        need(f.f != nullptr, AW_ERR_STATE, ("checkpoint: cannot open " + path + " for writing").c_str());
        write_header(f, h);
        AW_CUDA(cudaStreamWaitEvent(w.s, w.taken, 0));
        const size_t total = w.used;
        const size_t nchunk = (total + kChunkBytes - 1) / kChunkBytes;
        auto issue = [&](size_t k) {
            const size_t off = k * kChunkBytes, len = std::min(kChunkBytes, total - off);
            AW_CUDA(cudaMemcpyAsync(w.pin[k & 1], static_cast<const char*>(w.snap) + off, len,
                                    cudaMemcpyDeviceToHost, w.s));
            AW_CUDA(cudaEventRecord(w.done[k & 1], w.s));
        };
        if (nchunk) issue(0);
        for (size_t k = 0; k < nchunk; ++k) {
            if (k + 1 < nchunk) issue(k + 1);         // the other buffer was written to the file already
            AW_CUDA(cudaEventSynchronize(w.done[k & 1]));
            const size_t off = k * kChunkBytes, len = std::min(kChunkBytes, total - off);
            f.put(w.pin[k & 1], len);
        }
        need(std::fflush(f.f) == 0, AW_ERR_STATE, "checkpoint: flush failed");
    } catch (const std::exception& e) {
        w.err = e.what();
    }
}

void join(Ctx& c) {
    CkWriter* w = c.ck;
    if (!w || !w->th.joinable()) return;
    w->th.join();
    if (!w->err.empty()) {
        const std::string e = w->err;
        w->err.clear();
        throw Error(AW_ERR_STATE, e);
    }
}

}  // namespace

void free_checkpoint(Ctx& c) {
    CkWriter* w = c.ck;
    if (!w) return;
    if (w->th.joinable()) w->th.join();
    if (w->snap) cudaFree(w->snap);
    for (int k = 0; k < 2; ++k) {
        if (w->pin[k]) cudaFreeHost(w->pin[k]);
        if (w->done[k]) cudaEventDestroy(w->done[k]);
    }
    if (w->taken) cudaEventDestroy(w->taken);
    if (w->s) cudaStreamDestroy(w->s);
    delete w;
    c.ck = nullptr;
}

void checkpoint_write(Ctx& c, const std::string& path, const aw_checkpoint_info& info, bool wait) {
    need(c.parts.x != nullptr, AW_ERR_STATE, "particles not bound");
    need(c.inited, AW_ERR_STATE, "checkpoint: aw_init first");
    join(c);                                        // one write in flight at a time
    prepare_step(c);                                // acc_src holds the deposit of the current state
    if (!c.ck) c.ck = new CkWriter();
    CkWriter& w = *c.ck;
    writer_resources(w);
    Header h;
    h.seed = info.rng_seed; h.step = info.step; h.time = info.time; h.sd = info.sd; h.eps_l = info.eps_l;
    h.deck = info.deck ? info.deck : "";
    h.git = info.git_hash ? info.git_hash : "";
    h.manifest = arrays_of(c);
    size_t total = 0;
    for (const Arr& a : h.manifest) total += a.bytes();
    if (total > w.cap) {
        if (w.snap) AW_CUDA(cudaFree(w.snap));
        w.snap = nullptr;
        w.cap = 0;
        AW_CUDA(cudaMalloc(&w.snap, total));
        w.cap = total;
    }
    w.used = total;
    // the snapshot, in stream order with the run
    size_t off = 0;
    for (const Arr& a : h.manifest) {
        AW_CUDA(cudaMemcpyAsync(static_cast<char*>(w.snap) + off, a.dev, a.bytes(), cudaMemcpyDeviceToDevice,
                                c.stream));
        off += a.bytes();
    }
    AW_CUDA(cudaEventRecord(w.taken, c.stream));
    int device = 0;
    AW_CUDA(cudaGetDevice(&device));
    w.th = std::thread([&w, device, path, h]() { stream_out(w, device, path, h); });
    if (wait) join(c);
}

void checkpoint_wait(Ctx& c) { join(c); }

void checkpoint_read(Ctx& c, const std::string& path, aw_checkpoint_info* out) {
    need(c.parts.x != nullptr, AW_ERR_STATE, "particles not bound");
    join(c);
    File f;
    f.f = std::fopen(path.c_str(), "rb");
    need(f.f != nullptr, AW_ERR_ARG, ("checkpoint: cannot open " + path).c_str());
    const Header h = read_header(f);
    const std::vector<Arr> want = arrays_of(c);
    // where each wanted array sits in the payload
    std::vector<long long> at(want.size(), -1);
    long long off = 0;
    for (const Arr& m : h.manifest) {
        for (size_t i = 0; i < want.size(); ++i)
            if (want[i].name == m.name) {
                need(m.dtype == want[i].dtype && m.count == want[i].count, AW_ERR_ARG,
                     ("checkpoint: array '" + m.name + "' does not match this context (dtype or count)").c_str());
                at[i] = off;
            }
        off += static_cast<long long>(m.bytes());
    }
    for (size_t i = 0; i < want.size(); ++i)
        need(at[i] >= 0 || !required(want[i].name), AW_ERR_ARG,
             ("checkpoint: array '" + want[i].name + "' missing from the file").c_str());
    const long long base = std::ftell(f.f);
    need(base >= 0, AW_ERR_STATE, "checkpoint: cannot tell the file position");
    if (!c.ck) c.ck = new CkWriter();
    writer_resources(*c.ck);
    char* pin = static_cast<char*>(c.ck->pin[0]);
    AW_CUDA(cudaStreamSynchronize(c.stream));
    for (size_t i = 0; i < want.size(); ++i) {
        if (at[i] < 0) continue;
        need(std::fseek(f.f, static_cast<long>(base + at[i]), SEEK_SET) == 0, AW_ERR_STATE,
             "checkpoint: seek failed");
        const size_t total = want[i].bytes();
        for (size_t o = 0; o < total; o += kChunkBytes) {
            const size_t len = std::min(kChunkBytes, total - o);
            f.get(pin, len);
            AW_CUDA(cudaMemcpyAsync(static_cast<char*>(want[i].dev) + o, pin, len, cudaMemcpyHostToDevice,
                                    c.stream));
            AW_CUDA(cudaStreamSynchronize(c.stream));   // the pinned buffer is reused
        }
    }
    c.pending_valid = true;                          // acc_src holds the deposit of the restored state
    c.inited = true;
    c.host_step = h.step;
    if (out) {
        out->rng_seed = h.seed; out->step = h.step; out->time = h.time; out->sd = h.sd; out->eps_l = h.eps_l;
        out->deck = nullptr; out->git_hash = nullptr;
    }
}

}  // namespace aw
