// Host-side inputs for the exploration step: the ID-format dataset reader and the
// user-defined plan (.fmt) reader.
//
// * wk_load_id_dir reads a dataset directory as the POSIX loader does: every entry whose name
//   starts with "id_" (dot entries skipped, posix_loader.hpp:49-70), in sorted path order
//   (base_loader.hpp:235-237), each read as whitespace-separated decimal "s p o" triples until
//   the first token that is not one (the `while (file >> s >> p >> o)` loop,
//   base_loader.hpp:242-247).  One server holds every triple, so the partition filter keeps
//   them all.  The result goes to wk_gstore_build, which does the loader's sort and dedup.
// * wk_plan_apply_fmt orders and orients a pattern group by a .fmt text as
//   Planner::set_plan / set_direction do (planner.hpp:667-699, 723-770).
#include <dirent.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/wukong_b200.h"

namespace {

// One file's triples, appended to `out`.  A token that is not a decimal number in [0, 2^32)
// ends the file, as a failed extraction ends the reference's read loop; so does the end of
// the file, and a triple cut short there is dropped.
int read_id_file(const std::string& path, std::vector<uint32_t>& out) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return WK_E_BADARG;
    std::vector<char> buf(1 << 20);
    std::string tok;
    uint32_t tri[3];
    int k = 0;
    bool stop = false;
    auto take = [&]() {
        if (tok.empty()) return;
        bool ok = tok.size() <= 10;
        for (char c : tok) ok = ok && c >= '0' && c <= '9';
        const unsigned long long v = ok ? std::strtoull(tok.c_str(), nullptr, 10) : 0;
        if (!ok || v > 0xFFFFFFFFull) {
            stop = true;
        } else {
            tri[k++] = (uint32_t)v;
            if (k == 3) {
                out.insert(out.end(), tri, tri + 3);
                k = 0;
            }
        }
        tok.clear();
    };
    size_t got;
    while (!stop && (got = std::fread(buf.data(), 1, buf.size(), f)) > 0) {
        for (size_t i = 0; i < got && !stop; ++i) {
            const char c = buf[i];
            if (std::isspace((unsigned char)c)) take();
            else tok.push_back(c);
        }
    }
    if (!stop) take();
    std::fclose(f);
    return WK_SUCCESS;
}

std::string trim(const std::string& s) {
    size_t b = 0, e = s.size();
    while (b < e && std::isspace((unsigned char)s[b])) ++b;
    while (e > b && std::isspace((unsigned char)s[e - 1])) --e;
    return s.substr(b, e - b);
}

bool starts_with_ci(const std::string& s, const char* p) {
    for (size_t i = 0; p[i]; ++i)
        if (i >= s.size() || std::tolower((unsigned char)s[i]) != p[i]) return false;
    return true;
}

}  // namespace

extern "C" int wk_load_id_dir(const char* dir, uint32_t** triples, uint64_t* n_triples) {
    if (!dir || !triples || !n_triples) return WK_E_BADARG;
    *triples = nullptr;
    *n_triples = 0;
    std::string src(dir);
    if (src.empty()) return WK_E_BADARG;
    if (src.back() != '/') src.push_back('/');
    DIR* d = opendir(src.c_str());
    if (!d) return WK_E_BADARG;
    std::vector<std::string> files;
    while (struct dirent* ent = readdir(d)) {
        if (ent->d_name[0] == '.') continue;
        if (std::strncmp(ent->d_name, "id_", 3) == 0) files.push_back(src + ent->d_name);
    }
    closedir(d);
    std::sort(files.begin(), files.end());
    std::vector<uint32_t> all;
    for (const std::string& f : files) {
        const int rc = read_id_file(f, all);
        if (rc) return rc;
    }
    const uint64_t n = all.size() / 3;
    uint32_t* t = (uint32_t*)std::malloc(std::max<size_t>(all.size(), 1) * sizeof(uint32_t));
    if (!t) return WK_E_OOM;
    std::memcpy(t, all.data(), all.size() * sizeof(uint32_t));
    *triples = t;
    *n_triples = n;
    return WK_SUCCESS;
}

extern "C" int wk_plan_apply_fmt(const wk_pattern* patterns, int32_t n_patterns, const char* fmt_text,
                                 wk_pattern* out, int32_t out_cap, int32_t* n_out) {
    if ((!patterns && n_patterns) || n_patterns < 0 || !fmt_text || (!out && out_cap) || out_cap < 0 ||
        !n_out)
        return WK_E_BADARG;
    *n_out = 0;
    std::vector<long long> orders;
    std::vector<std::string> dirs;
    long long order = 0;
    std::string dir = ">";   // a line without a direction keeps the previous one
    const char* p = fmt_text;
    while (*p) {
        const char* e = std::strchr(p, '\n');
        std::string line(p, e ? (size_t)(e - p) : std::strlen(p));
        p = e ? e + 1 : p + line.size();
        line = trim(line);
        if (line.empty() || line[0] == '#' || line == "{") continue;
        if (line == "}") break;
        if (starts_with_ci(line, "union") || starts_with_ci(line, "optional"))
            return WK_E_UNSUPPORTED;   // nested groups are not on this path
        // `iss >> order >> dir`: a line that does not start with a number stores order 0,
        // which names no pattern and is refused below
        char* endp = nullptr;
        errno = 0;
        const long long v = std::strtoll(line.c_str(), &endp, 10);
        if (endp == line.c_str() || errno) {
            order = 0;
        } else {
            order = v;
            std::string rest = trim(std::string(endp));
            if (!rest.empty()) {
                const size_t sp = rest.find_first_of(" \t\r\f\v");
                dir = rest.substr(0, sp);
            }
        }
        orders.push_back(order);
        dirs.push_back(dir);
    }
    if ((long long)orders.size() < n_patterns) return WK_E_BADARG;   // "wrong format file content"
    if ((long long)orders.size() > out_cap) return WK_E_CAPACITY;
    for (size_t i = 0; i < orders.size(); ++i) {
        if (orders[i] < 1 || orders[i] > n_patterns) return WK_E_BADARG;
        wk_pattern q = patterns[orders[i] - 1];
        if (dirs[i] == "<") {
            q.direction = WK_IN;
            std::swap(q.subject, q.object);
        } else if (dirs[i] == ">") {
            q.direction = WK_OUT;
        } else if (dirs[i] == "<<") {
            q.direction = WK_IN;
            q.object = q.subject;
            q.subject = q.predicate;
            q.predicate = WK_PREDICATE_ID;
        } else if (dirs[i] == ">>") {
            q.direction = WK_OUT;
            q.subject = q.predicate;
            q.predicate = WK_PREDICATE_ID;
        }
        out[i] = q;
    }
    *n_out = (int32_t)orders.size();
    return WK_SUCCESS;
}
