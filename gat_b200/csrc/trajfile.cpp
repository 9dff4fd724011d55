/* The reference's formatted trajectory file (PreProcess::writeTraDataToFile and
 * readTraFromFormatedFile, PreProcess.cpp:203-315), host code:
 *
 *   line 1   the number of trajectories n
 *   line 2   xmin,ymin,xmax,ymax                      (printf %f)
 *   line 3   len_1;len_2;...;len_n;
 *   line 3+t one record per point of trajectory t:   lat,lon,tid,time;   (lat first; %f,%f,%d,%d)
 *
 * The writer reproduces the reference's bytes: std::to_chars in fixed notation with 6 digits
 * writes what printf's %f writes for the same double (the C++ standard defines it so), and the
 * trajectory lines are formatted on several threads and written in order. The reader loads the
 * file once, finds the line breaks, and parses the trajectory lines on several threads; each
 * field is parsed as strtod / strtol would parse it over the whole line (std::from_chars to
 * double, then float, after the leading blanks and '+' that strtod also skips; hexadecimal
 * numbers go to strtod itself). The reference copies each line into an unterminated buffer and
 * runs strtok past its end; here every line is checked against the lengths of line 3. */
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <charconv>
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <string_view>
#include <thread>
#include <vector>

#include "gat_b200.h"

namespace {

unsigned worker_count() { return std::max(1u, std::min(32u, std::thread::hardware_concurrency())); }

/* the whole file; false when it cannot be read */
bool slurp(const char* path, std::string& out) {
    FILE* f = fopen(path, "rb");
    if (!f) return false;
    bool ok = fseek(f, 0, SEEK_END) == 0;
    const long size = ok ? ftell(f) : -1;
    ok = ok && size >= 0 && fseek(f, 0, SEEK_SET) == 0;
    if (ok) {
        out.resize((size_t)size);
        ok = size == 0 || fread(&out[0], 1, (size_t)size, f) == (size_t)size;
    }
    fclose(f);
    return ok;
}

/* the first max_lines lines as std::getline splits them (a final line without '\n' counts when it
 * is not empty), one trailing '\r' removed */
void split_lines(const std::string& buf, size_t max_lines, std::vector<std::string_view>& lines) {
    const char* p = buf.data();
    const char* e = p + buf.size();
    while (lines.size() < max_lines && p < e) {
        const char* nl = static_cast<const char*>(memchr(p, '\n', (size_t)(e - p)));
        const char* le = nl ? nl : e;
        size_t len = (size_t)(le - p);
        if (len > 0 && p[len - 1] == '\r') len--;
        lines.emplace_back(p, len);
        p = nl ? nl + 1 : e;
    }
}

inline const char* skip_blank(const char* p, const char* e) {
    while (p < e && isspace((unsigned char)*p)) p++;
    return p;
}

/* one number as strtod reads it; false when none starts at p. *p advances past it. */
bool parse_double(const char*& p, const char* e, double* v) {
    const char* q = skip_blank(p, e);
    const char* s = q;
    bool neg = false;
    if (q < e && (*q == '+' || *q == '-')) {
        neg = *q == '-';
        q++;
    }
    /* strtod takes one sign; from_chars would accept a second '-' after the one stripped here */
    if (q < e && (*q == '+' || *q == '-')) return false;
    if (q + 1 < e && q[0] == '0' && (q[1] == 'x' || q[1] == 'X')) {
        /* hexadecimal: strtod itself, on a terminated copy of the token */
        const char* t = q;
        while (t < e && *t != ',' && *t != ';' && !isspace((unsigned char)*t)) t++;
        std::string tok(s, t);
        char* end = nullptr;
        const double d = strtod(tok.c_str(), &end);
        if (end == tok.c_str()) return false;
        *v = d;
        p = s + (end - tok.c_str());
        return true;
    }
    double d = 0;
    const std::from_chars_result r = std::from_chars(q, e, d);
    if (r.ptr == q) return false;
    /* out of range: strtod returns +-HUGE_VAL or a denormal/zero; from_chars leaves d alone */
    if (r.ec == std::errc::result_out_of_range) {
        std::string tok(q, r.ptr);
        d = strtod(tok.c_str(), nullptr);
    }
    *v = neg ? -d : d;
    p = r.ptr;
    return true;
}

/* one base-10 integer as strtol reads it (saturating on overflow) */
bool parse_long(const char*& p, const char* e, long* v) {
    const char* q = skip_blank(p, e);
    bool neg = false;
    if (q < e && (*q == '+' || *q == '-')) {
        neg = *q == '-';
        q++;
    }
    unsigned long u = 0;
    const std::from_chars_result r = std::from_chars(q, e, u);
    if (r.ptr == q) return false;
    if (r.ec == std::errc::result_out_of_range || (!neg && u > (unsigned long)LONG_MAX) ||
        (neg && u > (unsigned long)LONG_MAX + 1ul))
        *v = neg ? LONG_MIN : LONG_MAX;
    else
        *v = neg ? (long)(0ul - u) : (long)u;
    p = r.ptr;
    return true;
}

/* header: n, box, lengths; total points */
int parse_header(const std::vector<std::string_view>& lines, int* n, float box[4], std::vector<int32_t>* len,
                 int64_t* points) {
    if (lines.size() < 3) return GAT_ERR_ARG;
    const char* p = lines[0].data();
    long nn = 0;
    if (!parse_long(p, p + lines[0].size(), &nn) || nn < 0 || nn > (1L << 30)) return GAT_ERR_ARG;
    p = lines[1].data();
    const char* e = p + lines[1].size();
    for (int i = 0; i < 4; i++) {
        double v = 0;
        if (!parse_double(p, e, &v)) return GAT_ERR_ARG;
        if (box) box[i] = (float)v;
        if (i < 3) {
            if (p >= e || *p != ',') return GAT_ERR_ARG;
            p++;
        }
    }
    len->assign((size_t)nn, 0);
    p = lines[2].data();
    e = p + lines[2].size();
    int64_t total = 0;
    for (long t = 0; t < nn; t++) {
        long v = 0;
        if (!parse_long(p, e, &v) || v < 0 || v > (1L << 30) || p >= e || *p != ';') return GAT_ERR_ARG;
        (*len)[(size_t)t] = (int32_t)v;
        total += v;
        p++;
    }
    *n = (int)nn;
    *points = total;
    return GAT_OK;
}

/* parses trajectory line t (lat,lon,tid,time; records) into the arrays at offset o */
bool parse_line(std::string_view line, int L, int64_t o, float* lon, float* lat, int32_t* times) {
    const char* p = line.data();
    const char* e = p + line.size();
    for (int i = 0; i < L; i++, o++) {
        double la = 0, lo = 0;
        long tid = 0, tm = 0;
        if (!parse_double(p, e, &la) || p >= e || *p != ',') return false;
        p++;
        if (!parse_double(p, e, &lo) || p >= e || *p != ',') return false;
        p++;
        /* the point's trajectory id: the line number already says it */
        if (!parse_long(p, e, &tid) || p >= e || *p != ',') return false;
        p++;
        if (!parse_long(p, e, &tm) || p >= e || *p != ';') return false;
        p++;
        lat[o] = (float)la;
        lon[o] = (float)lo;
        if (times) times[o] = (int32_t)tm;
    }
    return true;
}

/* contiguous trajectory ranges of about equal point counts, one per worker */
std::vector<int> balance(const int32_t* lengths, int n, unsigned parts) {
    int64_t total = 0;
    for (int t = 0; t < n; t++) total += lengths[t];
    std::vector<int> cut{0};
    int64_t run = 0;
    for (int t = 0; t < n && cut.size() < parts; t++) {
        run += lengths[t];
        if (run * (int64_t)parts >= total * (int64_t)cut.size() && t + 1 < n) cut.push_back(t + 1);
    }
    cut.push_back(n);
    return cut;
}

inline void put_fixed6(std::string& s, float v) {
    char b[352];
    const std::to_chars_result r = std::to_chars(b, b + sizeof b, (double)v, std::chars_format::fixed, 6);
    s.append(b, (size_t)(r.ptr - b));
}
inline void put_int(std::string& s, long v) {
    char b[24];
    const std::to_chars_result r = std::to_chars(b, b + sizeof b, v);
    s.append(b, (size_t)(r.ptr - b));
}

}  // namespace

extern "C" {

int gat_traj_file_info(const char* path, int* n, int64_t* points, float box[4]) {
    if (!path || !n || !points) return GAT_ERR_ARG;
    /* the header only: read until three lines are complete */
    FILE* f = fopen(path, "rb");
    if (!f) return GAT_ERR_ARG;
    std::string buf;
    char chunk[1 << 16];
    int newlines = 0;
    size_t got;
    while (newlines < 3 && (got = fread(chunk, 1, sizeof chunk, f)) > 0) {
        buf.append(chunk, got);
        newlines += (int)std::count(chunk, chunk + got, '\n');
    }
    fclose(f);
    std::vector<std::string_view> lines;
    split_lines(buf, 3, lines);
    std::vector<int32_t> len;
    return parse_header(lines, n, box, &len, points);
}

int gat_traj_file_read(const char* path, int n, int64_t points, int32_t* lengths, float* lon, float* lat,
                       int32_t* times) {
    if (!path || n < 0 || points < 0 || (n > 0 && !lengths) || (points > 0 && (!lon || !lat))) return GAT_ERR_ARG;
    std::string buf;
    if (!slurp(path, buf)) return GAT_ERR_ARG;
    std::vector<std::string_view> lines;
    split_lines(buf, (size_t)n + 3, lines);
    int fn = 0;
    int64_t fp = 0;
    std::vector<int32_t> len;
    int st = parse_header(lines, &fn, nullptr, &len, &fp);
    if (st != GAT_OK) return st;
    if (fn != n || fp != points) return GAT_ERR_TRUNCATED; /* sizes from gat_traj_file_info */
    if (lines.size() < (size_t)n + 3) return GAT_ERR_ARG;
    std::vector<int64_t> off((size_t)n + 1, 0);
    for (int t = 0; t < n; t++) {
        lengths[t] = len[(size_t)t];
        off[(size_t)t + 1] = off[(size_t)t] + len[(size_t)t];
    }
    const std::vector<int> cut = balance(len.data(), n, worker_count());
    std::vector<char> ok(cut.size(), 1);
    std::vector<std::thread> th;
    for (size_t w = 0; w + 1 < cut.size(); w++)
        th.emplace_back([&, w]() {
            for (int t = cut[w]; t < cut[w + 1]; t++)
                if (!parse_line(lines[(size_t)t + 3], len[(size_t)t], off[(size_t)t], lon, lat, times)) {
                    ok[w] = 0;
                    return;
                }
        });
    for (auto& x : th) x.join();
    for (char c : ok)
        if (!c) return GAT_ERR_ARG;
    return GAT_OK;
}

int gat_traj_file_write(const char* path, int n, const int32_t* lengths, const float* lon, const float* lat,
                        const int32_t* times, const float box[4]) {
    if (!path || n < 0 || (n > 0 && (!lengths || !lon || !lat)) || !box) return GAT_ERR_ARG;
    for (int t = 0; t < n; t++)
        if (lengths[t] < 0) return GAT_ERR_ARG;
    FILE* f = fopen(path, "w");
    if (!f) return GAT_ERR_ARG;
    fprintf(f, "%d\n", n);
    fprintf(f, "%f,%f,%f,%f\n", box[0], box[1], box[2], box[3]);
    {
        std::string s;
        s.reserve((size_t)n * 4 + 2);
        for (int t = 0; t < n; t++) {
            put_int(s, lengths[t]);
            s.push_back(';');
        }
        s.push_back('\n');
        fwrite(s.data(), 1, s.size(), f);
    }
    std::vector<int64_t> off((size_t)n + 1, 0);
    for (int t = 0; t < n; t++) off[(size_t)t + 1] = off[(size_t)t] + lengths[t];
    /* rounds of one batch per worker, each about kBatch points, written in order */
    constexpr int64_t kBatch = 1 << 20;
    const unsigned nw = worker_count();
    std::vector<std::string> out(nw);
    int t0 = 0;
    while (t0 < n) {
        std::vector<std::pair<int, int>> ranges;
        int t = t0;
        for (unsigned w = 0; w < nw && t < n; w++) {
            const int s = t;
            int64_t pts = 0;
            while (t < n && (pts == 0 || pts + lengths[t] <= kBatch)) pts += lengths[t++];
            ranges.emplace_back(s, t);
        }
        std::vector<std::thread> th;
        for (size_t w = 0; w < ranges.size(); w++)
            th.emplace_back([&, w]() {
                std::string& s = out[w];
                s.clear();
                for (int u = ranges[w].first; u < ranges[w].second; u++) {
                    for (int64_t o = off[(size_t)u]; o < off[(size_t)u + 1]; o++) {
                        put_fixed6(s, lat[o]);
                        s.push_back(',');
                        put_fixed6(s, lon[o]);
                        s.push_back(',');
                        put_int(s, u + 1);
                        s.push_back(',');
                        put_int(s, times ? times[o] : 0);
                        s.push_back(';');
                    }
                    s.push_back('\n');
                }
            });
        for (auto& x : th) x.join();
        for (size_t w = 0; w < ranges.size(); w++) fwrite(out[w].data(), 1, out[w].size(), f);
        t0 = t;
    }
    const bool ok = !ferror(f);
    return (fclose(f) == 0 && ok) ? GAT_OK : GAT_ERR_ARG;
}

}  // extern "C"
