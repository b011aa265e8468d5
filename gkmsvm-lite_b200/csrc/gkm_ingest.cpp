// gkm_ingest.cpp -- the support-vector section of an LS-GKM model file parsed
// natively (importers/lsgkm.py:68-85 and importers/__init__.py:53-113 of
// gkmsvm-lite): lines "<coefficient> <sequence>" become float64 coefficients
// and one zero-padded [n, width] array of base codes (A C G T = 0..3; N and,
// counted for the caller's warning, any other letter stored as A) with each
// SV's length, ready for the device packing.  Host code: one pass to size the
// arrays, one to fill them.
#include <cerrno>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>

#include "gkm_b200.h"

int gkm_fail(int code, const char *fmt, ...);  // gkm_abi.cu

namespace {

struct CodeTable {
    uint8_t c[256];
    CodeTable()
    {
        memset(c, 5, sizeof(c));  // 5: not a DNA letter
        const char *b = "ACGT";
        for (int i = 0; i < 4; i++) {
            c[(uint8_t)b[i]] = (uint8_t)i;
            c[(uint8_t)(b[i] + ('a' - 'A'))] = (uint8_t)i;
        }
        c[(uint8_t)'N'] = c[(uint8_t)'n'] = 4;
    }
};
const CodeTable kCodes;

// str.split() separators of ASCII text
inline bool is_space(uint8_t ch) { return ch == ' ' || (ch >= '\t' && ch <= '\r') || (ch >= 0x1c && ch <= 0x1f); }

}  // namespace

extern "C" int gkm_lsgkm_parse_svs(const char *text, int64_t len, int64_t capacity, int64_t width, double *coef,
                                   int64_t *lengths, uint8_t *codes, int64_t *n_sv, int64_t *max_len,
                                   int64_t *n_other, int64_t *bad_line)
{
    if ((!text && len > 0) || len < 0 || !n_sv || !max_len)
        return gkm_fail(GKM_ERR_INVALID, "null argument or negative length");
    const bool fill = codes != nullptr;
    if (fill && (!coef || !lengths || capacity < 0 || width < 0))
        return gkm_fail(GKM_ERR_INVALID, "fill needs coef, lengths and codes");
    if (bad_line) *bad_line = -1;
    int64_t n = 0, longest = 0, other = 0, line_no = 0;
    const uint8_t *p = (const uint8_t *)text, *end = p + len;
    while (p < end) {
        const uint8_t *eol = (const uint8_t *)memchr(p, '\n', (size_t)(end - p));
        if (!eol) eol = end;
        line_no++;
        const uint8_t *q = p;
        p = eol + 1;
        while (q < eol && is_space(*q)) q++;
        if (q == eol) continue;  // blank line
        // a line starting "SV" is a section marker, skipped like the reference does
        if (eol - q >= 2 && q[0] == 'S' && q[1] == 'V') continue;
        const uint8_t *t0 = q;
        while (q < eol && !is_space(*q)) q++;
        const uint8_t *t1 = q;
        while (q < eol && is_space(*q)) q++;
        const uint8_t *s0 = q;
        while (q < eol && !is_space(*q)) q++;
        const uint8_t *s1 = q;
        if (s0 == s1) {
            if (bad_line) *bad_line = line_no;
            return gkm_fail(GKM_ERR_INVALID, "Malformed SV line %lld", (long long)line_no);
        }
        const int64_t L = s1 - s0;
        if (fill) {
            if (n >= capacity || L > width) return gkm_fail(GKM_ERR_INVALID, "SV section changed between passes");
            std::string tok((const char *)t0, (size_t)(t1 - t0));
            char *stop = nullptr;
            errno = 0;
            double v = strtod(tok.c_str(), &stop);
            if (stop != tok.c_str() + tok.size()) {
                if (bad_line) *bad_line = line_no;
                return gkm_fail(GKM_ERR_INVALID, "Malformed coefficient on SV line %lld", (long long)line_no);
            }
            coef[n] = v;
            lengths[n] = L;
            uint8_t *row = codes + n * width;
            bool odd = false;
            for (int64_t i = 0; i < L; i++) {
                const uint8_t ch = s0[i];
                if (ch >= 0x80) {
                    if (bad_line) *bad_line = line_no;
                    return gkm_fail(GKM_ERR_INVALID, "Non-ASCII letter on SV line %lld", (long long)line_no);
                }
                const uint8_t c = kCodes.c[ch];
                odd |= c == 5;
                row[i] = c > 3 ? 0 : c;
            }
            memset(row + L, 0, (size_t)(width - L));
            other += odd;
        }
        if (L > longest) longest = L;
        n++;
    }
    *n_sv = n;
    *max_len = longest;
    if (n_other) *n_other = other;
    return GKM_OK;
}
