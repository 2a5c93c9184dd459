// lsvd_autotune.cu -- per-size-class team shapes for the batched kernel.
//
// The batched planner asks for one ClassShape per size class.  Shapes come,
// in order of preference, from (1) the LSVD_SHAPES environment variable
// ("cls:nwarps,ts,g,per_team;..."), (2) the JSON cache written by
// lsvd_autotune_f64 (lsvd_api.cu; path LSVD_AUTOTUNE_CACHE, default
// $HOME/.cache/lsvd_b200/shapes.json): the "shapes_fp64" entry for the FP64
// kernel, a "shapes" entry for every precision, (3) the built-in defaults.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "lsvd_internal.h"

static bool parse_shapes(const char* s, ClassShape* shapes) {
    bool any = false;
    while (s && *s) {
        int c, w, ts, g, pt;
        int used = 0;
        if (std::sscanf(s, "%d:%d,%d,%d,%d%n", &c, &w, &ts, &g, &pt, &used) == 5) {
            if (c >= 0 && c < lsvd::kMaxClasses && (w == 0 || w == 1 || w == 2 || w == 4 || w == 8) &&
                (ts == 2 || ts == 4) && (g == 8 || g == 16 || g == 32) && pt >= 1 && pt <= 8) {
                shapes[c] = ClassShape{w, ts, g, pt};
                any = true;
            }
            s += used;
        } else {
            break;
        }
        while (*s == ';' || *s == ' ') ++s;
    }
    return any;
}

std::string lsvd_autotune_cache_path() {
    if (const char* p = std::getenv("LSVD_AUTOTUNE_CACHE")) return p;
    const char* home = std::getenv("HOME");
    return std::string(home ? home : "/tmp") + "/.cache/lsvd_b200/shapes.json";
}

void lsvd_autotune_shapes(lsvd_context* /*ctx*/, lsvd_precision prec, ClassShape* shapes) {
    for (int c = 0; c < lsvd::kMaxClasses; ++c) shapes[c] = lsvd_default_shape(c);
    if (prec != LSVD_PREC_FP64) {
        // the mixed path's FP32 tensor-core buffers are padded to 16: for
        // n in 17..32 two teams of four warps keep two CTAs per SM
        shapes[3] = ClassShape{4, 2, 8, 1};
        shapes[4] = ClassShape{4, 4, 8, 1};
    }
    // cache: one line {"shapes_fp64": "cls:w,ts,g,pt;...", ...}
    if (FILE* f = std::fopen(lsvd_autotune_cache_path().c_str(), "r")) {
        char buf[4096] = {0};
        size_t got = std::fread(buf, 1, sizeof(buf) - 1, f);
        std::fclose(f);
        buf[got] = 0;
        if (const char* q = std::strstr(buf, "\"shapes\": \"")) parse_shapes(q + 11, shapes);
        if (prec == LSVD_PREC_FP64)
            if (const char* q = std::strstr(buf, "\"shapes_fp64\": \"")) parse_shapes(q + 16, shapes);
    }
    if (const char* env = std::getenv("LSVD_SHAPES")) parse_shapes(env, shapes);
    shapes[0].nwarps = 0;  // micro class is always thread-per-matrix
}
