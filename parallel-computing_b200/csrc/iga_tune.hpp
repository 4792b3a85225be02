// Tuning table of the batched operator: rows per warp strip for each
// (degree, precision, size bucket) and warps per CTA for each (degree,
// precision), stored as a small JSON document.
#pragma once
#include <string>
#include <vector>

namespace iga {

struct TuneTable {
    struct Rows {
        int p = 0, prec = 0, ney_max = 0, rows = 0;
        double us = 0.0;
    };
    struct Warps {
        int p = 0, prec = 0, warps = 0;
        double us = 0.0;
    };
    std::string device;
    int sm_count = 0;
    std::vector<Rows> rows;
    std::vector<Warps> warps;
};

// Size buckets (element rows of the patch): the smallest bound >= ney.
int tune_bucket(int ney);

// Reads a table; a missing file gives an empty table and true. False (with a
// message) when the file exists but is not a valid table.
bool tune_read(const char *path, TuneTable &t, std::string &err);
bool tune_write(const char *path, const TuneTable &t, std::string &err);

// Rows per strip for a problem (0: no entry for its degree, precision and bucket).
int tune_rows(const TuneTable &t, int p, int prec, int ney);
// Warps per CTA for a degree (0: no entry).
int tune_warps(const TuneTable &t, int p, int prec);

void tune_set_rows(TuneTable &t, int p, int prec, int ney_max, int rows, double us);
void tune_set_warps(TuneTable &t, int p, int prec, int warps, double us);

}  // namespace iga
