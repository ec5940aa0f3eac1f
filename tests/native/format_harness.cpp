// Host build of pointvortex_b200/csrc/pv_format.cuh for the CPU tests: the same formatter source
// the GPU kernels run, compiled with g++ (tests/test_format.py builds it into a temporary
// directory).
#include "../../pointvortex_b200/csrc/pv_format.cuh"

#include <cstddef>

extern "C" {
// Formats values[i] into out + i * stride (NUL-terminated).
void pvf_format_many(const double *values, size_t n, char *out, size_t stride) {
    for (size_t i = 0; i < n; ++i) {
        char *o = out + i * stride;
        const int len = pvb::fmt::format_g17(values[i], o);
        o[len] = '\0';
    }
}
int pvf_format_u64(unsigned long long v, char *out) {
    const int len = pvb::fmt::format_u64(v, out);
    out[len] = '\0';
    return len;
}
}
