// WDM formatting and zstd framing (see wdm.hpp).
#include "wdm.hpp"

#include <dlfcn.h>

#include <algorithm>
#include <cstring>
#include <fstream>
#include <mutex>
#include <stdexcept>
#include <thread>

namespace bw {
namespace wdm {

namespace {

struct InBuf {
    const void* src;
    size_t size, pos;
};
struct OutBuf {
    void* dst;
    size_t size, pos;
};

// The few libzstd entry points the WDM contract needs, resolved from
// libzstd.so.1 at run time.  Parameter numbers are the stable public values
// (ZSTD_c_compressionLevel = 100, ZSTD_c_nbWorkers = 400, ZSTD_e_end = 2).
struct Zstd {
    void* h = nullptr;
    void* (*createCCtx)() = nullptr;
    size_t (*freeCCtx)(void*) = nullptr;
    size_t (*setParameter)(void*, int, int) = nullptr;
    size_t (*compressStream2)(void*, OutBuf*, InBuf*, int) = nullptr;
    size_t (*cstreamOutSize)() = nullptr;
    void* (*createDStream)() = nullptr;
    size_t (*freeDStream)(void*) = nullptr;
    size_t (*initDStream)(void*) = nullptr;
    size_t (*decompressStream)(void*, OutBuf*, InBuf*) = nullptr;
    size_t (*dstreamInSize)() = nullptr;
    size_t (*dstreamOutSize)() = nullptr;
    unsigned (*isError)(size_t) = nullptr;
    const char* (*errorName)(size_t) = nullptr;

    Zstd() {
        h = dlopen("libzstd.so.1", RTLD_NOW | RTLD_LOCAL);
        if (!h) return;
        auto get = [&](auto& fn, const char* name) { fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name)); };
        get(createCCtx, "ZSTD_createCCtx");
        get(freeCCtx, "ZSTD_freeCCtx");
        get(setParameter, "ZSTD_CCtx_setParameter");
        get(compressStream2, "ZSTD_compressStream2");
        get(cstreamOutSize, "ZSTD_CStreamOutSize");
        get(createDStream, "ZSTD_createDStream");
        get(freeDStream, "ZSTD_freeDStream");
        get(initDStream, "ZSTD_initDStream");
        get(decompressStream, "ZSTD_decompressStream");
        get(dstreamInSize, "ZSTD_DStreamInSize");
        get(dstreamOutSize, "ZSTD_DStreamOutSize");
        get(isError, "ZSTD_isError");
        get(errorName, "ZSTD_getErrorName");
    }
    bool ok() const {
        return h && createCCtx && freeCCtx && setParameter && compressStream2 && cstreamOutSize && createDStream &&
               freeDStream && initDStream && decompressStream && dstreamInSize && dstreamOutSize && isError &&
               errorName;
    }
    void check(size_t code, const char* what) const {
        if (isError(code)) throw std::runtime_error(std::string(what) + ": " + errorName(code));
    }
};

const Zstd& zstd() {
    static Zstd z;
    if (!z.ok()) throw std::runtime_error("libzstd.so.1 is not available (needed for .zst WDM files)");
    return z;
}

bool ends_with(const std::string& s, const std::string& suf) {
    return s.size() >= suf.size() && s.compare(s.size() - suf.size(), suf.size(), suf) == 0;
}

const unsigned char kMagic[4] = {0x28, 0xb5, 0x2f, 0xfd};

inline char* put_u64(char* p, uint64_t v) {
    char tmp[24];
    int n = 0;
    do {
        tmp[n++] = static_cast<char>('0' + v % 10);
        v /= 10;
    } while (v);
    while (n) *p++ = tmp[--n];
    return p;
}

// One text line: values[i*stride + offset] for i < count, space separated.
std::string format_line(const uint32_t* base, size_t count, size_t stride, uint32_t prime, bool canonicalise) {
    std::string out;
    out.resize(count * 11 + 1);
    char* p = out.data();
    for (size_t i = 0; i < count; ++i) {
        if (i) *p++ = ' ';
        uint32_t v = base[i * stride];
        if (canonicalise) v %= prime;
        p = put_u64(p, v);
    }
    *p++ = '\n';
    out.resize(static_cast<size_t>(p - out.data()));
    return out;
}

// Streaming token reader over a (possibly zstd) file.
class TokenReader {
public:
    explicit TokenReader(const std::string& path) : file_(path, std::ios::binary) {
        if (!file_) throw std::runtime_error("Failed to open file: " + path);
        unsigned char head[4] = {0, 0, 0, 0};
        file_.read(reinterpret_cast<char*>(head), 4);
        const bool compressed = file_.gcount() == 4 && std::memcmp(head, kMagic, 4) == 0;
        file_.clear();
        file_.seekg(0);
        if (compressed) {
            const Zstd& z = zstd();
            ds_ = z.createDStream();
            if (!ds_) throw std::runtime_error("Failed to allocate zstd decompression stream");
            z.check(z.initDStream(ds_), "Failed to initialize zstd decompression stream");
            in_.resize(z.dstreamInSize());
            out_.resize(z.dstreamOutSize());
        } else {
            out_.resize(1 << 20);
        }
    }
    ~TokenReader() {
        if (ds_) zstd().freeDStream(ds_);
    }
    // Next whitespace-separated unsigned integer; false at end of data.
    bool next_u64(uint64_t& v, const char* label) {
        int c;
        do {
            c = get();
        } while (c == ' ' || c == '\n' || c == '\t' || c == '\r');
        if (c < 0) return false;
        if (c < '0' || c > '9') throw std::runtime_error(std::string("Failed to read ") + label + " from WDM file");
        v = 0;
        while (c >= '0' && c <= '9') {
            v = v * 10 + static_cast<uint64_t>(c - '0');
            c = get();
        }
        return true;
    }
    uint64_t need_u64(const char* label) {
        uint64_t v;
        if (!next_u64(v, label)) throw std::runtime_error(std::string("Failed to read ") + label + " from WDM file");
        return v;
    }

private:
    int get() {
        if (pos_ == len_ && !refill()) return -1;
        return static_cast<unsigned char>(out_[pos_++]);
    }
    bool refill() {
        pos_ = len_ = 0;
        if (!ds_) {
            file_.read(out_.data(), static_cast<std::streamsize>(out_.size()));
            len_ = static_cast<size_t>(file_.gcount());
            return len_ > 0;
        }
        const Zstd& z = zstd();
        while (len_ == 0) {
            if (in_pos_ == in_len_) {
                if (frame_done_) return false;
                file_.read(in_.data(), static_cast<std::streamsize>(in_.size()));
                in_len_ = static_cast<size_t>(file_.gcount());
                in_pos_ = 0;
                if (in_len_ == 0) {
                    if (!frame_done_) throw std::runtime_error("Compressed WDM ended before the zstd frame was complete");
                    return false;
                }
            }
            InBuf ib{in_.data(), in_len_, in_pos_};
            OutBuf ob{out_.data(), out_.size(), 0};
            size_t ret = z.decompressStream(ds_, &ob, &ib);
            z.check(ret, "zstd decompression failed");
            in_pos_ = ib.pos;
            len_ = ob.pos;
            if (ret == 0) {
                frame_done_ = true;
                if (len_ == 0) return false;
            }
        }
        return true;
    }
    std::ifstream file_;
    void* ds_ = nullptr;
    std::vector<char> in_, out_;
    size_t in_pos_ = 0, in_len_ = 0, pos_ = 0, len_ = 0;
    bool frame_done_ = false;
};

}  // namespace

bool zstd_available() {
    static Zstd z;
    return z.ok();
}

void write_file(const std::string& path, const std::string& text) {
    std::ofstream out(path, std::ios::binary);
    if (!out) throw std::runtime_error("Failed to open file: " + path);
    if (!(ends_with(path, ".zst") || ends_with(path, ".zst.tmp"))) {
        out.write(text.data(), static_cast<std::streamsize>(text.size()));
    } else {
        const Zstd& z = zstd();
        void* cctx = z.createCCtx();
        if (!cctx) throw std::runtime_error("Failed to allocate zstd compression stream");
        try {
            z.check(z.setParameter(cctx, 100, 3), "Failed to initialize zstd compression stream");
            const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
            if (text.size() > (8u << 20) && hw > 1) {
                // Multithreaded frames where libzstd supports them; single-threaded otherwise.
                size_t r = z.setParameter(cctx, 400, static_cast<int>(std::min(hw, 16u)));
                (void)r;
            }
            std::vector<char> buf(z.cstreamOutSize());
            InBuf ib{text.data(), text.size(), 0};
            size_t remaining = 1;
            while (remaining != 0) {
                OutBuf ob{buf.data(), buf.size(), 0};
                remaining = z.compressStream2(cctx, &ob, &ib, 2 /* ZSTD_e_end */);
                z.check(remaining, "zstd compression failed");
                out.write(buf.data(), static_cast<std::streamsize>(ob.pos));
            }
        } catch (...) {
            z.freeCCtx(cctx);
            throw;
        }
        z.freeCCtx(cctx);
    }
    out.flush();
    if (!out) throw std::runtime_error("Failed to write WDM stream");
}

std::string read_file(const std::string& path) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("Failed to open file: " + path);
    std::string raw((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    if (raw.size() < 4 || std::memcmp(raw.data(), kMagic, 4) != 0) return raw;
    const Zstd& z = zstd();
    void* ds = z.createDStream();
    if (!ds) throw std::runtime_error("Failed to allocate zstd decompression stream");
    std::string out;
    try {
        z.check(z.initDStream(ds), "Failed to initialize zstd decompression stream");
        std::vector<char> buf(z.dstreamOutSize());
        InBuf ib{raw.data(), raw.size(), 0};
        size_t ret = 1;
        while (ib.pos < ib.size) {
            OutBuf ob{buf.data(), buf.size(), 0};
            ret = z.decompressStream(ds, &ob, &ib);
            z.check(ret, "zstd decompression failed");
            out.append(buf.data(), ob.pos);
            if (ret == 0 && ib.pos != ib.size) throw std::runtime_error("Compressed WDM has trailing bytes after zstd frame");
        }
        while (ret != 0) {   // flush what the decoder still holds
            OutBuf ob{buf.data(), buf.size(), 0};
            ret = z.decompressStream(ds, &ob, &ib);
            z.check(ret, "zstd decompression failed");
            if (ob.pos == 0 && ret != 0) throw std::runtime_error("Compressed WDM ended before the zstd frame was complete");
            out.append(buf.data(), ob.pos);
        }
    } catch (...) {
        z.freeDStream(ds);
        throw;
    }
    z.freeDStream(ds);
    return out;
}

std::string format_sym(size_t n_rows, size_t n_cols, uint32_t prime, size_t num_v,
                       const std::vector<uint32_t>& row_precond, const std::vector<uint32_t>& col_precond,
                       const std::vector<uint32_t>& initial, const std::vector<uint32_t>& current,
                       const std::vector<uint32_t>& packed, size_t nlen) {
    if (nlen == 0) throw std::runtime_error("Cannot save WDM file with empty sequence list");
    const size_t sp = num_v * (num_v + 1) / 2;
    if (row_precond.size() != n_rows || col_precond.size() != n_cols || initial.size() != n_cols * num_v ||
        current.size() != n_cols * num_v || packed.size() < nlen * sp)
        throw std::runtime_error("WDM buffers do not match the header dimensions");
    struct Job {
        const uint32_t* base;
        size_t count, stride;
        bool canon;
    };
    std::vector<Job> jobs;
    jobs.push_back({row_precond.data(), n_rows, 1, false});
    jobs.push_back({col_precond.data(), n_cols, 1, false});
    for (size_t v = 0; v < num_v; ++v) jobs.push_back({initial.data() + v, n_cols, num_v, true});
    for (size_t v = 0; v < num_v; ++v) jobs.push_back({current.data() + v, n_cols, num_v, true});
    for (size_t s = 0; s < sp; ++s) jobs.push_back({packed.data() + s, nlen, sp, true});
    std::vector<std::string> lines(jobs.size());
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const unsigned nt = std::min<unsigned>(hw, static_cast<unsigned>(jobs.size()));
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t)
        pool.emplace_back([&, t] {
            for (size_t j = t; j < jobs.size(); j += nt)
                lines[j] = format_line(jobs[j].base, jobs[j].count, jobs[j].stride, prime, jobs[j].canon);
        });
    for (auto& th : pool) th.join();
    std::string text = std::to_string(n_rows) + " " + std::to_string(n_cols) + " " + std::to_string(prime) + " " +
                       std::to_string(nlen) + " " + std::to_string(num_v) + "\n";
    size_t total = text.size();
    for (auto& l : lines) total += l.size();
    text.reserve(total);
    for (auto& l : lines) text += l;
    return text;
}

InitialState read_initial_state(const std::string& path) {
    TokenReader rd(path);
    InitialState st;
    st.rows = rd.need_u64("matrix row count");
    st.cols = rd.need_u64("matrix column count");
    st.prime = static_cast<uint32_t>(rd.need_u64("prime"));
    st.nlen = rd.need_u64("sequence length");
    st.num_v = rd.need_u64("vector count");
    st.row_precond.resize(st.rows);
    for (auto& v : st.row_precond) v = static_cast<uint32_t>(rd.need_u64("row preconditioner entry"));
    st.col_precond.resize(st.cols);
    for (auto& v : st.col_precond) v = static_cast<uint32_t>(rd.need_u64("column preconditioner entry"));
    st.initial_rowmajor.assign(st.cols * st.num_v, 0);
    for (size_t v = 0; v < st.num_v; ++v)
        for (size_t i = 0; i < st.cols; ++i)
            st.initial_rowmajor[i * st.num_v + v] = static_cast<uint32_t>(rd.need_u64("initial vector entry"));
    return st;
}

}  // namespace wdm
}  // namespace bw
