/* The reference's formatted trajectory file (PreProcess::writeTraDataToFile and
 * readTraFromFormatedFile, PreProcess.cpp:203-315), host code:
 *
 *   line 1   the number of trajectories n
 *   line 2   xmin,ymin,xmax,ymax                      (printf %f)
 *   line 3   len_1;len_2;...;len_n;
 *   line 3+t one record per point of trajectory t:   lat,lon,tid,time;   (lat first; %f,%f,%d,%d)
 *
 * The writer reproduces the reference's bytes. The reader parses every field with strtod /
 * strtol over the whole line (the reference copies each line into an unterminated buffer and
 * runs strtok past its end) and checks each line against the lengths of line 3. */
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

#include "gat_b200.h"

namespace {

bool read_lines(const char* path, std::vector<std::string>& lines, size_t max_lines) {
    std::ifstream in(path, std::ios::in | std::ios::binary);
    if (!in) return false;
    std::string s;
    while (lines.size() < max_lines && std::getline(in, s)) {
        if (!s.empty() && s.back() == '\r') s.pop_back();
        lines.push_back(s);
    }
    return true;
}

/* header: n, box, lengths; total points */
int parse_header(const std::vector<std::string>& lines, int* n, float box[4], std::vector<int32_t>* len, int64_t* points) {
    if (lines.size() < 3) return GAT_ERR_ARG;
    char* end = nullptr;
    errno = 0;
    long nn = strtol(lines[0].c_str(), &end, 10);
    if (errno || end == lines[0].c_str() || nn < 0 || nn > (1L << 30)) return GAT_ERR_ARG;
    const char* p = lines[1].c_str();
    for (int i = 0; i < 4; i++) {
        double v = strtod(p, &end);
        if (end == p) return GAT_ERR_ARG;
        if (box) box[i] = (float)v;
        p = end;
        if (i < 3) {
            if (*p != ',') return GAT_ERR_ARG;
            p++;
        }
    }
    len->assign((size_t)nn, 0);
    p = lines[2].c_str();
    int64_t total = 0;
    for (long t = 0; t < nn; t++) {
        long v = strtol(p, &end, 10);
        if (end == p || v < 0 || v > (1L << 30) || *end != ';') return GAT_ERR_ARG;
        (*len)[(size_t)t] = (int32_t)v;
        total += v;
        p = end + 1;
    }
    *n = (int)nn;
    *points = total;
    return GAT_OK;
}

}  // namespace

extern "C" {

int gat_traj_file_info(const char* path, int* n, int64_t* points, float box[4]) {
    if (!path || !n || !points) return GAT_ERR_ARG;
    std::vector<std::string> lines;
    if (!read_lines(path, lines, 3)) return GAT_ERR_ARG;
    std::vector<int32_t> len;
    return parse_header(lines, n, box, &len, points);
}

int gat_traj_file_read(const char* path, int n, int64_t points, int32_t* lengths, float* lon, float* lat,
                       int32_t* times) {
    if (!path || n < 0 || points < 0 || (n > 0 && !lengths) || (points > 0 && (!lon || !lat))) return GAT_ERR_ARG;
    std::vector<std::string> lines;
    if (!read_lines(path, lines, (size_t)n + 3)) return GAT_ERR_ARG;
    int fn = 0;
    int64_t fp = 0;
    std::vector<int32_t> len;
    int st = parse_header(lines, &fn, nullptr, &len, &fp);
    if (st != GAT_OK) return st;
    if (fn != n || fp != points) return GAT_ERR_TRUNCATED; /* sizes from gat_traj_file_info */
    if (lines.size() < (size_t)n + 3) return GAT_ERR_ARG;
    int64_t o = 0;
    for (int t = 0; t < n; t++) {
        lengths[t] = len[(size_t)t];
        const char* p = lines[(size_t)t + 3].c_str();
        char* end = nullptr;
        for (int i = 0; i < len[(size_t)t]; i++, o++) {
            double la = strtod(p, &end);
            if (end == p || *end != ',') return GAT_ERR_ARG;
            p = end + 1;
            double lo = strtod(p, &end);
            if (end == p || *end != ',') return GAT_ERR_ARG;
            p = end + 1;
            strtol(p, &end, 10); /* the point's trajectory id: the line number already says it */
            if (end == p || *end != ',') return GAT_ERR_ARG;
            p = end + 1;
            long tm = strtol(p, &end, 10);
            if (end == p || *end != ';') return GAT_ERR_ARG;
            p = end + 1;
            lat[o] = (float)la;
            lon[o] = (float)lo;
            if (times) times[o] = (int32_t)tm;
        }
    }
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
    for (int t = 0; t < n; t++) fprintf(f, "%d;", lengths[t]);
    fprintf(f, "\n");
    int64_t o = 0;
    for (int t = 0; t < n; t++) {
        for (int i = 0; i < lengths[t]; i++, o++)
            fprintf(f, "%f,%f,%d,%d;", lat[o], lon[o], t + 1, times ? times[o] : 0);
        fprintf(f, "\n");
    }
    const bool ok = !ferror(f);
    return (fclose(f) == 0 && ok) ? GAT_OK : GAT_ERR_ARG;
}

}  // extern "C"
