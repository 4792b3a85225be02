// One part of a partitioned mesh (include/iga_part.h): reader and checks of
// the reference's partition files, and the part's ghosted MatMult on the GPU.
//
// File formats (the reference's, so that its preprocessor's output drops in):
//   info.txt (matrix_free/src/FileManager.cpp:375-448): "key: value" lines
//     p, q, Lx, Ly, nElemX, nElemY, part_num_1d, dim, base_name.
//   <base_name>_<rank>.txt (matrix_free/src/FileManager.cpp:3-69, 114-280):
//     "nlocalfunc: N", "nlocalelemx: N", "nlocalelemy: N", then sections
//     ID, ghostID, Dir, IEN, ElemSize1, ElemSize2, CP, NURBSExtraction1,
//     NURBSExtraction2, each a name line followed by one line of numbers.
// The partition geometry (matrix_free/src/Partition.cpp:23-92): the control
// points of a direction with m functions are cut into part_num_1d runs of
// ceil(m / part_num_1d) (the last one shorter); part i's elements start p/2
// before its first function (the first part's at 0) and end where the next
// part's begin; the partition numbering takes the parts in order (y outer,
// x inner) and each part's functions x fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/iga_part.h"
#include "iga_plan.hpp"

using namespace iga;

struct iga_part {
    iga_part_info info{};
    std::vector<int> ID, ghost, Dir, IEN;
    std::vector<double> h1, h2, CP, C1, C2;
    std::vector<int> blk2loc;
    std::vector<double> CPblock;
    // device state
    iga_plan *plan = nullptr;
    int *d_blk2loc = nullptr, *d_id = nullptr;
    double *d_xb = nullptr, *d_yb = nullptr;
    int sign = IGA_SIGN_REFERENCE, bc = IGA_BC_REFERENCE, device = 0;
};

namespace {

// Partition geometry of one direction with m functions, nelem elements,
// degree p, P parts.
struct Cuts {
    std::vector<int> count, fstart, estart, ecount;
    bool ok = false;
};

Cuts cuts(int m, int nelem, int p, int P)
{
    Cuts c;
    if (P < 1 || m < 1) return c;
    const int size = (m + P - 1) / P;
    c.count.assign(P, size);
    c.count[P - 1] = m - (P - 1) * size;
    c.fstart.assign(P, 0);
    c.estart.assign(P, 0);
    for (int i = 1; i < P; ++i) {
        c.fstart[i] = i * size;
        c.estart[i] = c.fstart[i] - p / 2;
    }
    c.ecount.assign(P, 0);
    for (int i = 0; i < P; ++i) c.ecount[i] = (i + 1 < P ? c.estart[i + 1] : nelem) - c.estart[i];
    c.ok = true;
    for (int i = 0; i < P; ++i) c.ok = c.ok && c.count[i] > 0 && c.ecount[i] > 0;
    return c;
}

bool read_lines(const char *path, std::vector<std::string> &lines, std::string &err)
{
    std::ifstream f(path);
    if (!f.is_open()) {
        err = std::string("cannot open ") + path;
        return false;
    }
    std::string l;
    while (std::getline(f, l)) {
        if (!l.empty() && l.back() == '\r') l.pop_back();
        lines.push_back(l);
    }
    return true;
}

template <typename T>
bool parse_numbers(const std::string &line, std::vector<T> &out)
{
    out.clear();
    std::istringstream ss(line);
    std::string tok;
    while (ss >> tok) {
        char *end = nullptr;
        if (sizeof(T) == sizeof(int)) {
            const long v = std::strtol(tok.c_str(), &end, 10);
            if (*end) return false;
            out.push_back((T)v);
        } else {
            const double v = std::strtod(tok.c_str(), &end);
            if (*end) return false;
            out.push_back((T)v);
        }
    }
    return true;
}

bool key_value(const std::string &line, std::string &key, std::string &value)
{
    const size_t c = line.find(": ");
    if (c == std::string::npos) return false;
    key = line.substr(0, c);
    value = line.substr(c + 2);
    return true;
}

int fail(iga_part *pt, const std::string &msg)
{
    set_error("iga_part_open: " + msg);
    delete pt;
    return IGA_ERR_ARG;
}

__global__ void part_gather_kernel(const double *__restrict__ xl, double *__restrict__ xb,
                                   const int *__restrict__ blk2loc, const int *__restrict__ id, long long nb, int bc)
{
    for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nb; b += (long long)gridDim.x * blockDim.x) {
        const int k = blk2loc[b];
        xb[b] = (bc == IGA_BC_IDENTITY && id[k] < 0) ? 0.0 : xl[k];
    }
}

__global__ void part_scatter_kernel(const double *__restrict__ yb, const double *__restrict__ xl,
                                    double *__restrict__ yl, const int *__restrict__ blk2loc,
                                    const int *__restrict__ id, long long nb, int nowned, int bc)
{
    for (long long b = blockIdx.x * (long long)blockDim.x + threadIdx.x; b < nb; b += (long long)gridDim.x * blockDim.x) {
        const int k = blk2loc[b];
        double v = yb[b];
        if (id[k] < 0) v = (bc == IGA_BC_IDENTITY && k < nowned) ? xl[k] : 0.0;
        yl[k] = v;
    }
}

}  // namespace

extern "C" {

int iga_part_open(const char *info_file, const char *part_file, int rank, iga_part **out)
{
    if (!info_file || !part_file || !out) return IGA_ERR_ARG;
    *out = nullptr;
    iga_part *pt = new iga_part();
    iga_part_info &I = pt->info;
    std::string err;
    std::vector<std::string> lines;
    if (!read_lines(info_file, lines, err)) return fail(pt, err);
    int seen = 0;
    for (const std::string &l : lines) {
        std::string k, v;
        if (!key_value(l, k, v)) continue;
        char *end = nullptr;
        const double d = std::strtod(v.c_str(), &end);
        const bool num = end != v.c_str();
        if (k == "p" && num) I.p = (int)d, seen |= 1;
        else if (k == "q" && num) I.q = (int)d, seen |= 2;
        else if (k == "Lx" && num) I.Lx = d, seen |= 4;
        else if (k == "Ly" && num) I.Ly = d, seen |= 8;
        else if (k == "nElemX" && num) I.nElemX = (int)d, seen |= 16;
        else if (k == "nElemY" && num) I.nElemY = (int)d, seen |= 32;
        else if (k == "part_num_1d" && num) I.part_num_1d = (int)d, seen |= 64;
        else if (k == "dim" && num) I.dim = (int)d, seen |= 128;
    }
    if (seen != 255) return fail(pt, std::string(info_file) + ": missing p, q, Lx, Ly, nElemX, nElemY, part_num_1d or dim");
    if (I.p < 1 || I.q < 1 || I.nElemX < 1 || I.nElemY < 1 || I.part_num_1d < 1 || I.dim != 2)
        return fail(pt, "info: invalid sizes (dim must be 2)");
    const int P = I.part_num_1d;
    if (rank < 0 || rank >= P * P) return fail(pt, "rank outside 0 .. part_num_1d^2 - 1");
    I.rank = rank;
    I.part_x = rank % P;
    I.part_y = rank / P;
    const int m = I.nElemX + I.p, n = I.nElemY + I.q;
    I.nfunc_global = (int64_t)m * n;
    const Cuts cx = cuts(m, I.nElemX, I.p, P), cy = cuts(n, I.nElemY, I.q, P);
    if (!cx.ok || !cy.ok) return fail(pt, "part_num_1d too large for the mesh (an empty part)");

    lines.clear();
    if (!read_lines(part_file, lines, err)) return fail(pt, err);
    I.nlocalfunc = I.nlocalelemx = I.nlocalelemy = -1;
    for (size_t i = 0; i < lines.size(); ++i) {
        const std::string &l = lines[i];
        std::string k, v;
        if (key_value(l, k, v)) {
            const int val = std::atoi(v.c_str());
            if (k == "nlocalfunc") I.nlocalfunc = val;
            else if (k == "nlocalelemx") I.nlocalelemx = val;
            else if (k == "nlocalelemy") I.nlocalelemy = val;
            continue;
        }
        if (i + 1 >= lines.size()) break;
        const std::string &data = lines[i + 1];
        bool ok = true, known = true;
        if (l == "ID") ok = parse_numbers(data, pt->ID);
        else if (l == "ghostID") ok = parse_numbers(data, pt->ghost);
        else if (l == "Dir") ok = parse_numbers(data, pt->Dir);
        else if (l == "IEN") ok = parse_numbers(data, pt->IEN);
        else if (l == "ElemSize1") ok = parse_numbers(data, pt->h1);
        else if (l == "ElemSize2") ok = parse_numbers(data, pt->h2);
        else if (l == "CP") ok = parse_numbers(data, pt->CP);
        else if (l == "NURBSExtraction1") ok = parse_numbers(data, pt->C1);
        else if (l == "NURBSExtraction2") ok = parse_numbers(data, pt->C2);
        else known = false;
        if (!ok) return fail(pt, std::string(part_file) + ": bad numbers in section " + l);
        if (known) ++i;
    }
    const int nlf = I.nlocalfunc, nlx = I.nlocalelemx, nly = I.nlocalelemy;
    const int ng = (int)pt->ghost.size(), nloc = (I.p + 1) * (I.q + 1);
    I.nghost = ng;
    const int px = I.part_x, py = I.part_y;
    if (nlf != cx.count[px] * cy.count[py]) return fail(pt, "nlocalfunc does not match the partition of info.txt");
    if (nlx != cx.ecount[px] || nly != cy.ecount[py])
        return fail(pt, "nlocalelemx / nlocalelemy do not match the partition of info.txt");
    const int nl = nlf + ng;
    if ((int)pt->ID.size() != nl || (int)pt->CP.size() != 2 * nl || (int)pt->IEN.size() != nlx * nly * nloc ||
        (int)pt->h1.size() != nlx || (int)pt->h2.size() != nly ||
        (int)pt->C1.size() != nlx * (I.p + 1) * (I.p + 1) || (int)pt->C2.size() != nly * (I.q + 1) * (I.q + 1))
        return fail(pt, "section sizes do not match nlocalfunc, ghostID and the element counts");
    I.elem_x0 = cx.estart[px];
    I.elem_y0 = cy.estart[py];
    I.block_m = nlx + I.p;
    I.block_n = nly + I.q;
    if ((long long)I.block_m * I.block_n != nl)
        return fail(pt, "local form is not the part's block of control points");
    // partition number of natural function (i, j)
    std::vector<long long> part_off(P * P + 1, 0);
    for (int jj = 0; jj < P; ++jj)
        for (int ii = 0; ii < P; ++ii)
            part_off[jj * P + ii + 1] = part_off[jj * P + ii] + (long long)cx.count[ii] * cy.count[jj];
    I.owned_offset = part_off[rank];
    const int size_x = cx.count[0], size_y = cy.count[0];
    auto number = [&](int i, int j) -> long long {
        const int qi = i / size_x, qj = j / size_y;
        return part_off[qj * P + qi] + (long long)(j - cy.fstart[qj]) * cx.count[qi] + (i - cx.fstart[qi]);
    };
    // block map from the local IEN: element (ii, jj), local basis a = jl (p+1) + il
    pt->blk2loc.assign(nl, -1);
    std::vector<int> loc_seen(nl, 0);
    for (int jj = 0; jj < nly; ++jj)
        for (int ii = 0; ii < nlx; ++ii)
            for (int jl = 0; jl <= I.q; ++jl)
                for (int il = 0; il <= I.p; ++il) {
                    const int k = pt->IEN[(size_t)(jj * nlx + ii) * nloc + jl * (I.p + 1) + il];
                    if (k < 0 || k >= nl) return fail(pt, "IEN entry outside the local form");
                    const int b = (jj + jl) * I.block_m + (ii + il);
                    if (pt->blk2loc[b] == -1) {
                        pt->blk2loc[b] = k;
                        if (loc_seen[k]++) return fail(pt, "IEN maps two block positions to one local entry");
                    } else if (pt->blk2loc[b] != k) {
                        return fail(pt, "IEN is not a structured element block");
                    }
                }
    for (int b = 0; b < nl; ++b)
        if (pt->blk2loc[b] < 0) return fail(pt, "a block position is not touched by the part's elements");
    // every local entry is the function the partition numbering says it is
    for (int b = 0; b < nl; ++b) {
        const int k = pt->blk2loc[b];
        const int gi = I.elem_x0 + b % I.block_m, gj = I.elem_y0 + b / I.block_m;
        const long long num = number(gi, gj);
        const long long expect = k < nlf ? I.owned_offset + k : (long long)pt->ghost[k - nlf];
        if (num != expect) return fail(pt, "owned / ghost numbering differs from the partition of info.txt");
        if (pt->ID[k] != -1 && pt->ID[k] != num) return fail(pt, "ID entry is neither -1 nor the function's number");
    }
    pt->CPblock.resize(2 * (size_t)nl);
    for (int b = 0; b < nl; ++b) {
        pt->CPblock[2 * b] = pt->CP[2 * (size_t)pt->blk2loc[b]];
        pt->CPblock[2 * b + 1] = pt->CP[2 * (size_t)pt->blk2loc[b] + 1];
    }
    *out = pt;
    return IGA_OK;
}

int iga_part_close(iga_part *pt)
{
    if (!pt) return IGA_OK;
    if (pt->plan) iga_plan_destroy(pt->plan);
    for (void *p : {(void *)pt->d_blk2loc, (void *)pt->d_id, (void *)pt->d_xb, (void *)pt->d_yb})
        if (p) cudaFree(p);
    delete pt;
    return IGA_OK;
}

int iga_part_get_info(const iga_part *pt, iga_part_info *info)
{
    if (!pt || !info) return IGA_ERR_ARG;
    *info = pt->info;
    return IGA_OK;
}

int iga_part_ghosts(const iga_part *pt, int64_t *ghosts)
{
    if (!pt || !ghosts) return IGA_ERR_ARG;
    for (size_t i = 0; i < pt->ghost.size(); ++i) ghosts[i] = pt->ghost[i];
    return IGA_OK;
}

int iga_part_block_map(const iga_part *pt, int32_t *block_to_local)
{
    if (!pt || !block_to_local) return IGA_ERR_ARG;
    std::copy(pt->blk2loc.begin(), pt->blk2loc.end(), block_to_local);
    return IGA_OK;
}

int iga_part_local_id(const iga_part *pt, int32_t *id)
{
    if (!pt || !id) return IGA_ERR_ARG;
    std::copy(pt->ID.begin(), pt->ID.end(), id);
    return IGA_OK;
}

int iga_part_mesh(const iga_part *pt, iga_mesh_desc *d)
{
    if (!pt || !d) return IGA_ERR_ARG;
    *d = iga_mesh_desc{};
    d->p = pt->info.p;
    d->q = pt->info.q;
    d->nElemX = pt->info.nlocalelemx;
    d->nElemY = pt->info.nlocalelemy;
    d->CP = pt->CPblock.data();
    d->C1 = pt->C1.data();
    d->C2 = pt->C2.data();
    d->h1 = pt->h1.data();
    d->h2 = pt->h2.data();
    return IGA_OK;
}

int iga_part_build(iga_part *pt, const iga_opts *opts)
{
    if (!pt || !opts) return IGA_ERR_ARG;
    if (opts->precision != IGA_FP64 || (opts->bc != IGA_BC_REFERENCE && opts->bc != IGA_BC_IDENTITY) ||
        (opts->sign != IGA_SIGN_REFERENCE && opts->sign != IGA_SIGN_SPD)) {
        set_error("iga_part_build: FP64, sign REFERENCE or SPD, bc REFERENCE or IDENTITY");
        return IGA_ERR_ARG;
    }
    if (pt->plan) {
        set_error("iga_part_build: already built");
        return IGA_ERR_ARG;
    }
    iga_mesh_desc d;
    iga_part_mesh(pt, &d);
    iga_opts o = *opts;
    o.bc = IGA_BC_NONE;
    int st = iga_plan_create(&d, &o, &pt->plan);
    if (st) return st;
    pt->sign = opts->sign;
    pt->bc = opts->bc;
    pt->device = opts->device;
    const size_t nl = pt->blk2loc.size();
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc((void **)&pt->d_blk2loc, sizeof(int) * nl);
    if (e == cudaSuccess) e = cudaMalloc((void **)&pt->d_id, sizeof(int) * nl);
    if (e == cudaSuccess) e = cudaMalloc((void **)&pt->d_xb, sizeof(double) * nl);
    if (e == cudaSuccess) e = cudaMalloc((void **)&pt->d_yb, sizeof(double) * nl);
    if (e == cudaSuccess) e = cudaMemcpy(pt->d_blk2loc, pt->blk2loc.data(), sizeof(int) * nl, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(pt->d_id, pt->ID.data(), sizeof(int) * nl, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        set_error(std::string("iga_part_build: ") + cudaGetErrorString(e));
        return e == cudaErrorMemoryAllocation ? IGA_ERR_NOMEM : IGA_ERR_CUDA;
    }
    return IGA_OK;
}

int iga_part_apply(iga_part *pt, const double *x_local, double *y_local, void *stream)
{
    if (!pt || !x_local || !y_local) return IGA_ERR_ARG;
    if (!pt->plan) {
        set_error("iga_part_apply: call iga_part_build first");
        return IGA_ERR_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const long long nb = (long long)pt->blk2loc.size();
    const int blocks = (int)std::min<long long>((nb + 255) / 256, 4 * 148);
    part_gather_kernel<<<blocks, 256, 0, s>>>(x_local, pt->d_xb, pt->d_blk2loc, pt->d_id, nb, pt->bc);
    int st = iga_apply_internal_sb(pt->plan, IGA_FP64, pt->d_xb, pt->d_yb, s, pt->sign, IGA_BC_NONE);
    if (st) return st;
    part_scatter_kernel<<<blocks, 256, 0, s>>>(pt->d_yb, x_local, y_local, pt->d_blk2loc, pt->d_id, nb,
                                               pt->info.nlocalfunc, pt->bc);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error(std::string("iga_part_apply: ") + cudaGetErrorString(e));
        return IGA_ERR_CUDA;
    }
    return IGA_OK;
}

}  // extern "C"
