// Residual history file (Residual.res) in the reference's two layouts.
//
// Euler3D (Euler3D/src/RMSIO.cpp:21-97): a header of rule lines and column
// names chosen by the solution variables and by whether a preconditioner is
// on, then one line per iteration: iteration, the RMS of each equation,
// RMS_Res, the time-step extrema, the eigenvalue extrema of lambda 1, 4, 5
// and, with a preconditioner, the extrema of its sigma; a closing rule line.
// MPFLOW3D (MPFLOW3D/src/RMSIO.cpp:21-154): the same, with each RMS also
// given normalised by the scale MPFLOW3D accumulates over its first five
// writes (1 for those five).
//
// The column names, widths and printf formats are the file format and are
// kept identical, so the file can replace the reference's; the lines are
// built here from a column table.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "cfd_internal.h"

struct cfd_rms_file {
    FILE *f = nullptr;
    int layout = CFD_RMSFILE_EULER3D;
    int precond = 0;
    int nsave = 0;
    double scale[5] = {0, 0, 0, 0, 0};
    double scale_res = 0.0;
    size_t width = 0;
};

namespace {

const char *const kVarsEuler3D[3][5] = {
    {"RMS_RHO", "RMS_RHOU", "RMS_RHOV", "RMS_RHOW", "RMS_E"},  // conservative
    {"RMS_P", "RMS_U", "RMS_V", "RMS_W", "RMS_T"},             // (p, u, v, w, T)
    {"RMS_RHO", "RMS_U", "RMS_V", "RMS_W", "RMS_P"},           // any other set
};
const char *const kVarsMpflow3D[4][5] = {
    {"RHO", "RHOU", "RHOV", "RHOW", "E"},
    {"RHO", "U", "V", "W", "P"},
    {"P", "U", "V", "W", "T"},
    {"RHO", "U", "V", "W", "T"},
};
const char *const kTail[] = {"MIN_TIME", "MAX_TIME", "MIN_LAMDA1", "MAX_LAMDA1", "MIN_LAMDA4",
                             "MAX_LAMDA4", "MIN_LAMDA5", "MAX_LAMDA5", "MIN_SIGMA", "MAX_SIGMA"};

// " Iter" then every name right-aligned in 12 columns.
std::string header_line(const std::vector<std::string> &names) {
    std::string s = " Iter";
    char buf[64];
    for (const auto &n : names) {
        std::snprintf(buf, sizeof buf, "%12s", n.c_str());
        s += buf;
    }
    return s;
}

}  // namespace

extern "C" {

int cfd_rms_file_open(const char *path, int layout, int variables, int precond, cfd_rms_file **out) {
    if (!path || !out || (layout != CFD_RMSFILE_EULER3D && layout != CFD_RMSFILE_MPFLOW3D) ||
        variables < CFD_VARS_CONSERVATIVE || variables > CFD_VARS_RUT) {
        cfd::set_error("cfd_rms_file_open: path, layout (CFD_RMSFILE_*) and variables (CFD_VARS_*)");
        return CFD_ERR_ARG;
    }
    std::vector<std::string> names;
    if (layout == CFD_RMSFILE_EULER3D) {
        const int set = variables == CFD_VARS_CONSERVATIVE ? 0 : variables == CFD_VARS_PUT ? 1 : 2;
        for (const char *n : kVarsEuler3D[set]) names.push_back(n);
    } else {
        for (const char *n : kVarsMpflow3D[variables]) names.push_back(std::string("RMS_S") + n);
        names.push_back("RMS_SRES");
        for (const char *n : kVarsMpflow3D[variables]) names.push_back(std::string("RMS_") + n);
    }
    names.push_back("RMS_RES");
    for (int k = 0; k < (precond ? 10 : 8); k++) names.push_back(kTail[k]);
    const std::string head = header_line(names);
    FILE *f = std::fopen(path, "wb");
    if (!f) {
        cfd::set_error("cfd_rms_file_open: cannot write %s", path);
        return CFD_ERR_IO;
    }
    auto *r = new cfd_rms_file;
    r->f = f;
    r->layout = layout;
    r->precond = precond ? 1 : 0;
    r->width = head.size();
    const std::string eq(r->width, '='), dash(r->width, '-');
    std::fprintf(f, "%s\n%s\n%s\n%s\n", eq.c_str(), dash.c_str(), head.c_str(), dash.c_str());
    std::fflush(f);
    *out = r;
    return CFD_OK;
}

int cfd_rms_file_write(cfd_rms_file *r, int iteration, const double rms[6], const double extrema[8],
                       const double sigma[2]) {
    if (!r || !r->f || !rms || !extrema || (r->precond && !sigma)) {
        cfd::set_error("cfd_rms_file_write: open file, rms[6], extrema[8] (and sigma[2] with a preconditioner)");
        return CFD_ERR_ARG;
    }
    std::vector<double> v;
    if (r->layout == CFD_RMSFILE_MPFLOW3D) {
        // MPFLOW3D's normalisation (RMSIO.cpp:119-137): the per-equation scale
        // sums the first five RMS values; the total's scale adds all five
        // equations' RMS and is divided by 10 at each of those writes
        double s[5], sres;
        if (r->nsave < 5) {
            for (int k = 0; k < 5; k++) {
                r->scale[k] += rms[k];
                r->scale_res += rms[k];
            }
            r->scale_res /= 10.0;
            r->nsave++;
        }
        if (r->nsave < 5) {
            for (int k = 0; k < 5; k++) s[k] = 1.0;
            sres = 1.0;
        } else {
            for (int k = 0; k < 5; k++) s[k] = rms[k] / r->scale[k];
            sres = rms[5] / r->scale_res;
        }
        v.assign(s, s + 5);
        v.push_back(sres);
    }
    v.insert(v.end(), rms, rms + 6);
    // {min dt, max dt, min/max lambda1, lambda4, lambda5} from cfd_get_extrema's order
    const double tail[8] = {extrema[6], extrema[7], extrema[0], extrema[1], extrema[2], extrema[3], extrema[4],
                            extrema[5]};
    v.insert(v.end(), tail, tail + 8);
    if (r->precond) v.insert(v.end(), sigma, sigma + 2);
    std::fprintf(r->f, "%5d", iteration);
    for (double x : v) std::fprintf(r->f, " %10.5e", x);
    std::fprintf(r->f, "\n");
    std::fflush(r->f);
    return std::ferror(r->f) ? CFD_ERR_IO : CFD_OK;
}

int cfd_rms_file_write_ctx(cfd_rms_file *r, cfd_ctx *ctx, int iteration, int include_diss) {
    if (!r || !ctx) return CFD_ERR_ARG;
    if (r->precond) {
        cfd::set_error("cfd_rms_file_write_ctx: the preconditioner's sigma extrema are not kept by the context; "
                       "use cfd_rms_file_write");
        return CFD_ERR_ARG;
    }
    double rms[6], ext[8];
    int st = cfd_residual_rms(ctx, include_diss, rms);
    if (st) return st;
    if ((st = cfd_get_extrema(ctx, ext))) return st;
    return cfd_rms_file_write(r, iteration, rms, ext, nullptr);
}

int cfd_rms_file_close(cfd_rms_file *r) {
    if (!r) return CFD_ERR_ARG;
    int st = CFD_OK;
    if (r->f) {
        const std::string eq(r->width, '=');
        std::fprintf(r->f, "%s\n", eq.c_str());
        if (std::fclose(r->f) != 0) st = CFD_ERR_IO;
    }
    delete r;
    return st;
}

}  // extern "C"
