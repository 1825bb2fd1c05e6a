// Host-side helpers shared by the three command-line drivers: the prefix-file
// formats of the reference pipeline, its cache-identity strings, exit-code
// mapping of the library's status codes, and a context holder.
//
// The drivers keep the reference's command lines, files and exit codes
// (tools/build_aknn_source.cpp, tools/dataset_gt.cpp, src/rknn_query.cpp) and
// run every compute stage through libanqi's C ABI (include/anqi.h).
#pragma once

#include "anqi.h"

#include <sys/resource.h>
#include <sys/stat.h>

#include <cctype>
#include <cerrno>
#include <cstdarg>
#include <cinttypes>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

namespace anqi_cli {

// A failure that ends the program with `code` after printing `msg` to stderr.
struct Exit : std::runtime_error {
    int code;
    Exit(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

[[noreturn]] inline void die(int code, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
inline void die(int code, const char* fmt, ...) {
    char buf[4096];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    throw Exit(code, buf);
}

// Library status -> process exit code.  2/3/5 are the reference's own codes;
// device failures (no reference counterpart) exit 7, 8 or 9 like the status.
inline int exit_code(int status) { return status; }

inline double peak_gb() {
    struct rusage usage {};
    getrusage(RUSAGE_SELF, &usage);
    return usage.ru_maxrss / 1e6;
}

// ------------------------------------------------------------------ context
class Device {
  public:
    explicit Device(const char* tag) : tag_(tag) {
        const int rc = anqi_ctx_create(0, &ctx_);
        if (rc != ANQI_OK) die(exit_code(rc), "%s no usable CUDA device (status %d)", tag_, rc);
    }
    ~Device() { anqi_ctx_destroy(ctx_); }
    Device(const Device&) = delete;
    Device& operator=(const Device&) = delete;
    anqi_ctx* get() const { return ctx_; }
    // Throws with the library's message when rc is not ANQI_OK.
    void check(int rc, const char* what) const {
        if (rc != ANQI_OK) die(exit_code(rc), "%s %s failed: %s", tag_, what, anqi_last_error(ctx_));
    }

  private:
    const char* tag_;
    anqi_ctx* ctx_ = nullptr;
};

// ------------------------------------------------------------- fbin vectors
// [u32 n][u32 d][n x d f32] with the reference's size check.
struct Fbin {
    uint32_t n = 0, d = 0;
    std::vector<float> x;
};

inline bool read_fbin(const std::string& path, Fbin& out, std::string& why) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f) {
        why = "cannot open";
        return false;
    }
    const std::streamoff bytes = f.tellg();
    f.seekg(0);
    if (bytes < 8 || !f.read(reinterpret_cast<char*>(&out.n), 4) || !f.read(reinterpret_cast<char*>(&out.d), 4) ||
        out.n == 0 || out.d == 0) {
        why = "invalid fbin header";
        return false;
    }
    const uint64_t values = (uint64_t)out.n * out.d;
    if (8 + values * 4 != (uint64_t)bytes) {
        why = "invalid fbin size";
        return false;
    }
    out.x.resize(values);
    if (!f.read(reinterpret_cast<char*>(out.x.data()), (std::streamsize)(values * 4))) {
        why = "cannot read fbin values";
        return false;
    }
    return true;
}

inline bool fbin_header(const std::string& path, uint32_t& n, uint32_t& d) {
    std::ifstream f(path, std::ios::binary);
    return f.read(reinterpret_cast<char*>(&n), 4) && f.read(reinterpret_cast<char*>(&d), 4);
}

inline void write_file_or_die(const std::string& path, const std::vector<std::pair<const void*, size_t>>& parts,
                              int code, const char* tag) {
    std::ofstream f(path, std::ios::binary | std::ios::trunc);
    for (const auto& p : parts) f.write(static_cast<const char*>(p.first), (std::streamsize)p.second);
    f.close();
    if (!f) die(code, "%s failed writing %s", tag, path.c_str());
}

// ------------------------------------------------------- identity strings
// FNV-1a 64 as 16 hex digits (src/rknn_query.cpp:202-206,236-243).
inline uint64_t fnv1a(const void* data, size_t len, uint64_t h = 1469598103934665603ull) {
    const unsigned char* p = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < len; i++) {
        h ^= (uint64_t)p[i];
        h *= 1099511628211ull;
    }
    return h;
}

inline std::string hex64(uint64_t v) {
    char buf[17];
    snprintf(buf, sizeof(buf), "%016llx", (unsigned long long)v);
    return buf;
}

inline std::string hash16(const std::string& s) { return hex64(fnv1a(s.data(), s.size())); }

// path:dev..:ino..:sz..:mt..:ct.. (src/rknn_query.cpp:226-234).
inline std::string file_stat_identity(const std::string& path) {
    struct stat st;
    if (::stat(path.c_str(), &st) != 0) return path + ":missing";
    return path + ":dev" + std::to_string((uint64_t)st.st_dev) + ":ino" + std::to_string((uint64_t)st.st_ino) +
           ":sz" + std::to_string((uint64_t)st.st_size) + ":mt" + std::to_string((int64_t)st.st_mtime) + ":ct" +
           std::to_string((int64_t)st.st_ctime);
}

// path:sz<bytes>:fnv<hash of the contents> (src/rknn_query.cpp:208-224).
inline std::string file_fingerprint(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return path + ":missing";
    uint64_t h = 1469598103934665603ull, bytes = 0;
    std::vector<char> buf(1 << 16);
    while (f) {
        f.read(buf.data(), (std::streamsize)buf.size());
        const std::streamsize got = f.gcount();
        h = fnv1a(buf.data(), (size_t)got, h);
        bytes += (uint64_t)got;
    }
    return path + ":sz" + std::to_string(bytes) + ":fnv" + hex64(h);
}

inline std::string sanitize_tag(std::string s) {
    for (char& c : s) {
        const bool ok = (c >= '0' && c <= '9') || (c >= 'a' && c <= 'z') || (c >= 'A' && c <= 'Z') || c == '-' ||
                        c == '_';
        if (!ok) c = '_';
    }
    return s;
}

inline std::string env_or(const char* k, const char* d) {
    const char* v = std::getenv(k);
    return (v && *v) ? std::string(v) : std::string(d);
}

inline bool env_flag(const char* k) {
    const char* v = std::getenv(k);
    if (!v || !*v) return false;
    std::string s(v);
    for (char& c : s) c = (char)std::tolower((unsigned char)c);
    return s != "0" && s != "false" && s != "no" && s != "off";
}

// mkdir -p (the run scripts create the cache directories this way).
inline void mkdir_p(const std::string& dir) {
    for (size_t i = 1; i <= dir.size(); i++)
        if (i == dir.size() || dir[i] == '/') ::mkdir(dir.substr(0, i).c_str(), 0700);
}

inline bool file_exists(const std::string& p) {
    std::ifstream f(p);
    return f.good();
}

// Positive integer with the reference's strictness (whole string, > 0).
inline bool parse_positive(const char* text, uint64_t& out) {
    if (!text || !*text) return false;
    char* end = nullptr;
    errno = 0;
    const unsigned long long v = std::strtoull(text, &end, 10);
    if (errno == ERANGE || end == text || *end != '\0' || v == 0) return false;
    out = v;
    return true;
}

// Non-negative integer (the build tool's optional arguments).
inline bool parse_count(const char* text, uint64_t& out) {
    if (!text || !*text || *text == '-') return false;
    char* end = nullptr;
    errno = 0;
    const unsigned long long v = std::strtoull(text, &end, 10);
    if (errno == ERANGE || end == text || *end != '\0') return false;
    out = v;
    return true;
}

// ---------------------------------------------------------------- .rec
// n x K x {u32 id, f32 key} (tools/build_aknn_source.cpp:118-130).
struct TopKRecord {
    uint32_t id;
    float key;
};
static_assert(sizeof(TopKRecord) == 8, "record layout");

// --------------------------------------------------------------- timing
inline void write_timing(const std::string& path, const std::string& header,
                         const std::vector<std::pair<std::string, std::string>>& fields, int code, const char* tag) {
    std::ofstream f(path);
    f << header << "\n";
    for (const auto& kv : fields) f << kv.first << " " << kv.second << "\n";
    f.close();
    if (!f) die(code, "%s failed writing %s", tag, path.c_str());
}

inline std::string g17(double v) {
    char buf[64];
    snprintf(buf, sizeof(buf), "%.17g", v);
    return buf;
}

}  // namespace anqi_cli
