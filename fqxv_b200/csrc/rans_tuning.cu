// Launch-shape parameters of a context and the tuning table that sets them.
//
// The reference picks nothing at run time but its SIMD backend
// (crates/fqxv-rans/src/lib.rs:80-97, Backend::detect). Here the launch
// shapes of the batched kernels are parameters of the context: the decoder
// of wide order-1 alphabets (one warp per stream, several streams per SM, or
// four warps per stream, one per SM) as a function of how many such streams
// a batch holds, the CTAs per SM of every decode class, the table-size edges
// that split dense order-1 streams into launch groups, and the encode
// kernel's grid. Their defaults are the run-time rules the library always
// had; a tuning table measured on the device (fqxv_b200/tune.py writes one)
// replaces them. The table is a flat JSON object of integer parameters; it is
// read from the file named by FQXV_RANS_TUNING, else from tuning/<device
// name>.json beside the package directory of the library, when present.
#include <dlfcn.h>

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "rans_ctx.cuh"

namespace fqxv {

namespace {

struct ParamDef {
    const char *name;
    int64_t Tuning::*field;
    int64_t lo, hi;
};

const ParamDef kParams[] = {
    {"o1_four_max_streams", &Tuning::o1_four_max_streams, -1, 1 << 30},
    {"o1_top_latency_pct", &Tuning::o1_top_latency_pct, 0, 100000},
    {"o1_top_max", &Tuning::o1_top_max, -1, 1 << 30},
    {"o1_top_exclusive", &Tuning::o1_top_exclusive, 0, 1},
    {"o1_top_small_per_sm", &Tuning::o1_top_small_per_sm, 1, 4},
    {"cta_cap_o0", &Tuning::cta_cap_o0, 1, 64},
    {"cta_cap_o1_small", &Tuning::cta_cap_o1_small, 1, 64},
    {"cta_cap_o1_wide", &Tuning::cta_cap_o1_wide, 1, 64},
    {"cta_cap_o1_four", &Tuning::cta_cap_o1_four, 1, 16},
    {"cta_cap_o1_global", &Tuning::cta_cap_o1_global, 1, 64},
    {"cta_cap_o1_small_topped", &Tuning::cta_cap_o1_small_topped, 1, 64},
    {"cta_cap_o1_wide_topped", &Tuning::cta_cap_o1_wide_topped, 1, 64},
    {"dense_edge_small", &Tuning::dense_edge_small, 0, kDenseImageMax},
    {"dense_edge_large", &Tuning::dense_edge_large, 0, kDenseImageMax},
    {"enc_run_ctas_per_sm", &Tuning::enc_run_ctas_per_sm, 1, 64},
    {"enc_run_ctas_per_sm_uniform", &Tuning::enc_run_ctas_per_sm_uniform, 1, 64},
    {"enc_o1_keys", &Tuning::enc_o1_keys, 0, 1},
    {"host_enc_chunks", &Tuning::host_enc_chunks, 1, 16},
    {"host_dec_chunks", &Tuning::host_dec_chunks, 1, 16},
    {"host_in_place", &Tuning::host_in_place, -1, 1},
    {"host_out_mirror", &Tuning::host_out_mirror, 0, 1},
};

// Integer value of "key" in a flat JSON object (no nesting inside values).
bool json_int(const std::string &text, const char *key, int64_t &out) {
    const std::string q = std::string("\"") + key + "\"";
    size_t p = text.find(q);
    if (p == std::string::npos) return false;
    p = text.find(':', p + q.size());
    if (p == std::string::npos) return false;
    p++;
    while (p < text.size() && std::isspace((unsigned char)text[p])) p++;
    char *end = nullptr;
    const long long v = std::strtoll(text.c_str() + p, &end, 10);
    if (end == text.c_str() + p) return false;
    out = (int64_t)v;
    return true;
}

bool read_file(const std::string &path, std::string &out) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    char buf[4096];
    size_t k;
    out.clear();
    while ((k = std::fread(buf, 1, sizeof buf, f)) > 0 && out.size() < (1 << 20)) out.append(buf, k);
    std::fclose(f);
    return true;
}

// "NVIDIA B200" -> "nvidia_b200"
std::string file_stem(const char *device_name) {
    std::string s;
    for (const char *c = device_name; *c; c++) s += std::isalnum((unsigned char)*c) ? (char)std::tolower(*c) : '_';
    return s;
}

}  // namespace

int tuning_set(Tuning &t, const char *key, int64_t value) {
    for (const auto &d : kParams) {
        if (std::strcmp(d.name, key) != 0) continue;
        if (value < d.lo || value > d.hi) return FQXV_RANS_E_INVALID_ARG;
        t.*d.field = value;
        return FQXV_RANS_OK;
    }
    return FQXV_RANS_E_INVALID_ARG;
}

int tuning_get(const Tuning &t, const char *key, int64_t &value) {
    for (const auto &d : kParams) {
        if (std::strcmp(d.name, key) != 0) continue;
        value = t.*d.field;
        return FQXV_RANS_OK;
    }
    return FQXV_RANS_E_INVALID_ARG;
}

// Applies every known parameter found in the JSON text; returns how many.
int tuning_apply_json(Tuning &t, const std::string &text) {
    int k = 0;
    for (const auto &d : kParams) {
        int64_t v;
        if (json_int(text, d.name, v) && tuning_set(t, d.name, v) == FQXV_RANS_OK) k++;
    }
    return k;
}

void tuning_load(Tuning &t, int device) {
    std::string path;
    if (const char *e = std::getenv("FQXV_RANS_TUNING")) {
        path = e;
    } else {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        Dl_info info;
        if (!dladdr(reinterpret_cast<void *>(&tuning_load), &info) || !info.dli_fname) return;
        std::string lib = info.dli_fname;  // .../fqxv_b200/_lib/libfqxv_rans_gpu.so
        const size_t a = lib.rfind('/');
        if (a == std::string::npos) return;
        const size_t b = lib.rfind('/', a - 1);
        if (b == std::string::npos) return;
        path = lib.substr(0, b) + "/tuning/" + file_stem(prop.name) + ".json";
    }
    std::string text;
    if (read_file(path, text)) {
        tuning_apply_json(t, text);
        t.source = path;
    }
}

}  // namespace fqxv
