// JSON tuning table of the batched operator (format "iga-batch-tune-1"):
//   {"format": "iga-batch-tune-1", "device": "...", "sm_count": 148,
//    "rows":  [{"p": 3, "precision": "fp64", "ney_max": 64, "rows_per_strip": 16, "us": 12.5}, ...],
//    "warps": [{"p": 3, "precision": "fp64", "warps": 7, "us": 80.1}, ...]}
// "precision" is "fp64" (FP64 batches) or "mixed" (the FP32 operator of
// mixed-precision batches). A minimal recursive-descent reader covers the
// JSON this writer emits (objects, arrays, strings without escapes beyond \"
// and \\, numbers, true/false/null).
#include "iga_tune.hpp"

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>

#include "../../include/iga_mf.h"

namespace iga {

namespace {

struct JVal {
    enum Kind { NUL, BOOL, NUM, STR, ARR, OBJ } kind = NUL;
    double num = 0.0;
    std::string str;
    std::vector<JVal> arr;
    std::vector<std::pair<std::string, JVal>> obj;
    const JVal *get(const char *k) const
    {
        for (const auto &kv : obj)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
};

struct Parser {
    const char *s, *e;
    std::string err;
    void ws()
    {
        while (s < e && std::isspace((unsigned char)*s)) ++s;
    }
    bool fail(const char *m)
    {
        if (err.empty()) err = m;
        return false;
    }
    bool str(std::string &out)
    {
        if (s >= e || *s != '"') return fail("expected string");
        ++s;
        out.clear();
        while (s < e && *s != '"') {
            if (*s == '\\') {
                ++s;
                if (s >= e) return fail("bad escape");
                if (*s != '"' && *s != '\\' && *s != '/') return fail("unsupported escape");
            }
            out.push_back(*s++);
        }
        if (s >= e) return fail("unterminated string");
        ++s;
        return true;
    }
    bool value(JVal &v, int depth)
    {
        if (depth > 16) return fail("nesting too deep");
        ws();
        if (s >= e) return fail("unexpected end");
        if (*s == '{') {
            ++s;
            v.kind = JVal::OBJ;
            ws();
            if (s < e && *s == '}') {
                ++s;
                return true;
            }
            for (;;) {
                ws();
                std::string k;
                if (!str(k)) return false;
                ws();
                if (s >= e || *s != ':') return fail("expected ':'");
                ++s;
                JVal c;
                if (!value(c, depth + 1)) return false;
                v.obj.emplace_back(k, std::move(c));
                ws();
                if (s < e && *s == ',') {
                    ++s;
                    continue;
                }
                if (s < e && *s == '}') {
                    ++s;
                    return true;
                }
                return fail("expected ',' or '}'");
            }
        }
        if (*s == '[') {
            ++s;
            v.kind = JVal::ARR;
            ws();
            if (s < e && *s == ']') {
                ++s;
                return true;
            }
            for (;;) {
                JVal c;
                if (!value(c, depth + 1)) return false;
                v.arr.push_back(std::move(c));
                ws();
                if (s < e && *s == ',') {
                    ++s;
                    continue;
                }
                if (s < e && *s == ']') {
                    ++s;
                    return true;
                }
                return fail("expected ',' or ']'");
            }
        }
        if (*s == '"') {
            v.kind = JVal::STR;
            return str(v.str);
        }
        if (e - s >= 4 && !std::strncmp(s, "true", 4)) {
            v.kind = JVal::BOOL;
            v.num = 1;
            s += 4;
            return true;
        }
        if (e - s >= 5 && !std::strncmp(s, "false", 5)) {
            v.kind = JVal::BOOL;
            s += 5;
            return true;
        }
        if (e - s >= 4 && !std::strncmp(s, "null", 4)) {
            s += 4;
            return true;
        }
        char *end = nullptr;
        const std::string tok(s, (size_t)std::min<ptrdiff_t>(e - s, 64));
        v.num = std::strtod(tok.c_str(), &end);
        if (end == tok.c_str()) return fail("unexpected character");
        v.kind = JVal::NUM;
        s += end - tok.c_str();
        return true;
    }
};

int prec_of(const std::string &s)
{
    if (s == "fp64") return IGA_FP64;
    if (s == "mixed") return IGA_MIXED;
    return -1;
}

const char *prec_name(int p) { return p == IGA_MIXED ? "mixed" : "fp64"; }

bool as_int(const JVal *v, int &out)
{
    if (!v || v->kind != JVal::NUM) return false;
    out = (int)v->num;
    return (double)out == v->num;
}

}  // namespace

int tune_bucket(int ney)
{
    static const int bounds[] = {32, 64, 96, 128, 192, 256, 384, 512, 1024, 2048, 4096};
    for (int b : bounds)
        if (ney <= b) return b;
    return 1 << 30;
}

bool tune_read(const char *path, TuneTable &t, std::string &err)
{
    t = TuneTable{};
    FILE *f = std::fopen(path, "rb");
    if (!f) return true;   // no table yet
    std::string text;
    char buf[4096];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) {
        text.append(buf, n);
        if (text.size() > (size_t(1) << 22)) {
            std::fclose(f);
            err = "tuning table larger than 4 MiB";
            return false;
        }
    }
    std::fclose(f);
    Parser ps{text.data(), text.data() + text.size(), {}};
    JVal root;
    if (!ps.value(root, 0)) {
        err = "tuning table: " + ps.err;
        return false;
    }
    ps.ws();
    if (ps.s != ps.e) {
        err = "tuning table: trailing characters";
        return false;
    }
    if (root.kind != JVal::OBJ) {
        err = "tuning table: not an object";
        return false;
    }
    const JVal *fmt = root.get("format");
    if (!fmt || fmt->kind != JVal::STR || fmt->str != "iga-batch-tune-1") {
        err = "tuning table: missing or unknown format";
        return false;
    }
    if (const JVal *d = root.get("device"))
        if (d->kind == JVal::STR) t.device = d->str;
    as_int(root.get("sm_count"), t.sm_count);
    auto entries = [&](const char *key) -> const JVal * {
        const JVal *a = root.get(key);
        return (a && a->kind == JVal::ARR) ? a : nullptr;
    };
    if (const JVal *a = entries("rows"))
        for (const JVal &v : a->arr) {
            TuneTable::Rows r;
            const JVal *pr = v.get("precision");
            if (v.kind != JVal::OBJ || !as_int(v.get("p"), r.p) || !as_int(v.get("ney_max"), r.ney_max) ||
                !as_int(v.get("rows_per_strip"), r.rows) || !pr || pr->kind != JVal::STR ||
                (r.prec = prec_of(pr->str)) < 0 || r.rows < 1 || r.p < 1) {
                err = "tuning table: bad rows entry";
                return false;
            }
            if (const JVal *us = v.get("us"))
                if (us->kind == JVal::NUM) r.us = us->num;
            t.rows.push_back(r);
        }
    if (const JVal *a = entries("warps"))
        for (const JVal &v : a->arr) {
            TuneTable::Warps w;
            const JVal *pr = v.get("precision");
            if (v.kind != JVal::OBJ || !as_int(v.get("p"), w.p) || !as_int(v.get("warps"), w.warps) || !pr ||
                pr->kind != JVal::STR || (w.prec = prec_of(pr->str)) < 0 || w.warps < 1 || w.p < 1) {
                err = "tuning table: bad warps entry";
                return false;
            }
            if (const JVal *us = v.get("us"))
                if (us->kind == JVal::NUM) w.us = us->num;
            t.warps.push_back(w);
        }
    return true;
}

bool tune_write(const char *path, const TuneTable &t, std::string &err)
{
    FILE *f = std::fopen(path, "wb");
    if (!f) {
        err = std::string("cannot write tuning table ") + path;
        return false;
    }
    std::string dev;
    for (char c : t.device)
        if (c != '"' && c != '\\') dev.push_back(c);
    std::fprintf(f, "{\n  \"format\": \"iga-batch-tune-1\",\n  \"device\": \"%s\",\n  \"sm_count\": %d,\n",
                 dev.c_str(), t.sm_count);
    std::fprintf(f, "  \"rows\": [");
    for (size_t i = 0; i < t.rows.size(); ++i) {
        const auto &r = t.rows[i];
        std::fprintf(f,
                     "%s\n    {\"p\": %d, \"precision\": \"%s\", \"ney_max\": %d, \"rows_per_strip\": %d, \"us\": %.3f}",
                     i ? "," : "", r.p, prec_name(r.prec), r.ney_max, r.rows, r.us);
    }
    std::fprintf(f, "\n  ],\n  \"warps\": [");
    for (size_t i = 0; i < t.warps.size(); ++i) {
        const auto &w = t.warps[i];
        std::fprintf(f, "%s\n    {\"p\": %d, \"precision\": \"%s\", \"warps\": %d, \"us\": %.3f}", i ? "," : "", w.p,
                     prec_name(w.prec), w.warps, w.us);
    }
    std::fprintf(f, "\n  ]\n}\n");
    const bool ok = std::fclose(f) == 0;
    if (!ok) err = std::string("error writing ") + path;
    return ok;
}

int tune_rows(const TuneTable &t, int p, int prec, int ney)
{
    const int b = tune_bucket(ney);
    for (const auto &r : t.rows)
        if (r.p == p && r.prec == prec && r.ney_max == b) return r.rows;
    return 0;
}

int tune_warps(const TuneTable &t, int p, int prec)
{
    for (const auto &w : t.warps)
        if (w.p == p && w.prec == prec) return w.warps;
    return 0;
}

void tune_set_rows(TuneTable &t, int p, int prec, int ney_max, int rows, double us)
{
    for (auto &r : t.rows)
        if (r.p == p && r.prec == prec && r.ney_max == ney_max) {
            r.rows = rows;
            r.us = us;
            return;
        }
    t.rows.push_back({p, prec, ney_max, rows, us});
}

void tune_set_warps(TuneTable &t, int p, int prec, int warps, double us)
{
    for (auto &w : t.warps)
        if (w.p == p && w.prec == prec) {
            w.warps = warps;
            w.us = us;
            return;
        }
    t.warps.push_back({p, prec, warps, us});
}

}  // namespace iga
