/* Parameters of the PatchTable path: defaults, speed presets and switch parsing.

   Mirrors PatchTableParams (patchtable/patchtable_params.h:23-161) and its methods in
   patchtable/patchtable.cpp: set_defaults (:26-136), set_speed (:138-150), set_from_switches
   (:152-373).  Switch names, defaults and presets are the reference's so that command lines and
   callers carry over unchanged. */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "patchtable_b200.h"
#include "pt_internal.h"

namespace {

std::vector<std::string> split(const std::string &s, char c) {
    std::vector<std::string> out;
    std::string cur;
    for (char ch : s) {
        if (ch == c) { out.push_back(cur); cur.clear(); }
        else cur.push_back(ch);
    }
    out.push_back(cur);
    return out;
}

/* parse_switches, patchtable.cpp:9-19: "-name value" pairs; a later pair overrides.  Like the
   reference, argv[0] is never examined (it is the program name on a command line). */
std::map<std::string, std::string> parse_switches(const std::vector<std::string> &argv) {
    std::map<std::string, std::string> ans;
    for (size_t i = 1; i < argv.size(); i++) {
        if (!argv[i].empty() && argv[i][0] == '-' && i + 1 < argv.size()) {
            ans[argv[i]] = argv[i + 1];
            i += 1;
        }
    }
    return ans;
}

/* The speed presets, patchtable.cpp:139-148. */
const char *SPEED_PRESETS[10] = {
    "-ndims 8 -nchroma 1 -limit 10.000000 -do_rs 1 -run_dt 1 -partition_step 1 -dt_iters -1 -do_prop 1 -query_step 1 -kcoherence 20 -kcoherence_iter -1 -prop_iters 2 -spatial 1",
    "-ndims 6 -nchroma 1 -limit 100.000000 -do_rs 1 -run_dt 1 -partition_step 1 -dt_iters -1 -do_prop 1 -query_step 1 -kcoherence 10 -kcoherence_iter 0 -prop_iters 2 -spatial 1",
    "-ndims 6 -nchroma 1 -limit 100.000000 -do_rs 1 -run_dt 1 -partition_step 1 -dt_iters -1 -do_prop 1 -query_step 1 -kcoherence 10 -kcoherence_iter 0 -prop_iters 2 -spatial 0",
    "-ndims 6 -nchroma 1 -limit 100.000000 -do_rs 0 -run_dt 1 -partition_step 1 -dt_iters -1 -do_prop 1 -query_step 1 -kcoherence 2 -kcoherence_iter -1 -prop_iters 2 -spatial 0",
    "-ndims 7 -nchroma 1 -limit 10.000000 -do_rs 1 -run_dt 1 -partition_step 1 -dt_iters -1 -do_prop 1 -query_step 2 -kcoherence 20 -kcoherence_iter 0 -prop_iters 1 -spatial 1",
    "-ndims 8 -nchroma 1 -limit 100.000000 -do_rs 1 -run_dt 1 -partition_step 1 -dt_iters -1 -do_prop 1 -query_step 2 -kcoherence 4 -kcoherence_iter 0 -prop_iters 1 -spatial 1",
    "-ndims 6 -nchroma 1 -limit 100.000000 -do_rs 0 -run_dt 1 -partition_step 1 -dt_iters -1 -do_prop 1 -query_step 2 -kcoherence 2 -kcoherence_iter -1 -prop_iters 1 -spatial 0",
    "-ndims 7 -nchroma 1 -limit 1.000000 -do_rs 1 -run_dt 1 -partition_step 1 -dt_iters -1 -do_prop 1 -query_step 4 -kcoherence 3 -kcoherence_iter 0 -prop_iters 1 -spatial 1",
    "-ndims 6 -nchroma 1 -limit 100.000000 -do_rs 1 -run_dt 1 -partition_step 1 -dt_iters -1 -do_prop 1 -query_step 6 -kcoherence 5 -kcoherence_iter 0 -prop_iters 1 -spatial 0",
    "-ndims 6 -nchroma 1 -limit 100.000000 -do_rs 0 -run_dt 1 -partition_step 1 -dt_iters -1 -do_prop 1 -query_step 10 -kcoherence 5 -kcoherence_iter 0 -prop_iters 1 -spatial 0",
};

pt_status apply_switches(pt_params *p, const std::vector<std::string> &argv);

/* set_from_switches(string), patchtable.cpp:152-160: the string is split on spaces and handed
   over as an argv, so its first token takes the program-name slot and is ignored.  The speed
   presets start with -ndims, which is therefore never applied by set_speed. */
pt_status apply_string(pt_params *p, const std::string &s) {
    std::vector<std::string> L = split(s, ' '), argv;
    for (auto &t : L)
        if (!t.empty() && !(t.size() == 1 && t[0] == ' ')) argv.push_back(t);
    return apply_switches(p, argv);
}

int to_i(const std::string &s) { return atoi(s.c_str()); }
double to_f(const std::string &s) { return atof(s.c_str()); }

pt_status apply_switches(pt_params *p, const std::vector<std::string> &argv) {
    auto sw = parse_switches(argv);
    auto has = [&](const char *k) { return sw.count(k) > 0; };
    if (has("-speed")) {
        pt_status st = pt_params_set_speed(p, to_i(sw["-speed"]));
        if (st != PT_OK) return st;
    }
    if (has("-limit")) p->limit = (double) (int) (1000 * 1000 * to_f(sw["-limit"]));
#define INT_SW(name) if (has("-" #name)) p->name = to_i(sw["-" #name]);
#define BOOL_SW(name) if (has("-" #name)) p->name = to_i(sw["-" #name]) != 0;
#define DBL_SW(name) if (has("-" #name)) p->name = to_f(sw["-" #name]);
    BOOL_SW(randomize_dt) BOOL_SW(parallel_dt)
    INT_SW(threads) INT_SW(verbose)
    BOOL_SW(populate_nearest) BOOL_SW(populate_random)
    INT_SW(partition_step) INT_SW(ndims) INT_SW(nchroma) INT_SW(ntables)
    if (has("-nslices")) {
        std::vector<std::string> nL = split(sw["-nslices"], ',');
        if ((int) nL.size() > PT_MAX_DIMS) return pt_fail(PT_BAD_ARG, "-nslices has more than %d entries", PT_MAX_DIMS);
        p->ndims = (int) nL.size();
        p->n_nslices = (int) nL.size();
        for (size_t i = 0; i < nL.size(); i++) p->nslices[i] = to_i(nL[i]);
    }
    BOOL_SW(run_dt) BOOL_SW(do_prop) BOOL_SW(do_rs) INT_SW(spatial)
    if (has("-load")) snprintf(p->load_filename, PT_PATH_MAX, "%s", sw["-load"].c_str());
    if (has("-save")) snprintf(p->save_filename, PT_PATH_MAX, "%s", sw["-save"].c_str());
    INT_SW(patch_w)
    INT_SW(prop_iters) INT_SW(dt_iters) INT_SW(query_step)
    DBL_SW(coherence_spatial) DBL_SW(coherence_temporal) BOOL_SW(recalc_dist_temporal)
    if (has("-dt_algo")) {
        static const char *names[] = {"raster", "prop", "brute", "kdtree", "downsample", "hybrid", "euclidean"};
        int found = -1;
        for (int i = 0; i < 7; i++) if (sw["-dt_algo"] == names[i]) found = i;
        if (found < 0) return pt_fail(PT_BAD_ARG, "invalid dt_algo");
        p->dt_algo = found;
    }
    if (has("-colorspace")) {
        const std::string &m = sw["-colorspace"];
        if (m == "yuv") p->colorspace = 0;
        else if (m == "lab") p->colorspace = 1;
        else if (m == "rgb") p->convert_colorspace = 0;
        else return pt_fail(PT_BAD_ARG, "unsupported colorspace");
    }
    if (has("-lookup_algo")) {
        static const char *names[] = {"table", "brute", "kdtree", "pm", "treecann"};
        int found = -1;
        for (int i = 0; i < 5; i++) if (sw["-lookup_algo"] == names[i]) found = i;
        if (found < 0) return pt_fail(PT_BAD_ARG, "unsupported lookup_algo");
        p->lookup_algo = found;
    }
    if (has("-kcoherence_algo")) {
        static const char *names[] = {"flann", "pm", "ann", "treecann"};
        int found = -1;
        for (int i = 0; i < 4; i++) if (sw["-kcoherence_algo"] == names[i]) found = i;
        if (found < 0) return pt_fail(PT_BAD_ARG, "unsupported kcoherence_algo");
        p->kcoherence_algo = found;
    }
    if (has("-dim_algo")) {
        const std::string &m = sw["-dim_algo"];
        if (m == "pca") p->dim_algo = 1;
        else if (m == "wh") p->dim_algo = 0;
        else return pt_fail(PT_BAD_ARG, "unsupported dim_algo");
    }
    INT_SW(flann_reset_step) INT_SW(flann_build_step) INT_SW(query_iters)
    INT_SW(kcoherence) INT_SW(kcoherence_iter) INT_SW(kcoherence_min_dist) INT_SW(kcoherence_step)
    BOOL_SW(incoherence) DBL_SW(triangle_factor)
    BOOL_SW(init_random) BOOL_SW(sanitize_input) BOOL_SW(do_table_lookup)
    INT_SW(grid_ndims) DBL_SW(table_ratio) INT_SW(prop_dist)
    BOOL_SW(is_descriptor) BOOL_SW(descriptor_padded)
    INT_SW(gpu_prop_passes) INT_SW(gpu_jump) INT_SW(gpu_pull_max) INT_SW(gpu_tile)
    INT_SW(pca_samples) BOOL_SW(pca_mean) BOOL_SW(pca_subtract_mean) INT_SW(gpu_bands) INT_SW(gpu_kc_max)
#undef INT_SW
#undef BOOL_SW
#undef DBL_SW
    return PT_OK;
}

}  // namespace

extern "C" {

void pt_params_default(pt_params *p) {
    memset(p, 0, sizeof(*p));
    /* set_defaults, patchtable.cpp:26-136 (fields of the GPU path). */
    p->randomize_dt = 0;
    p->parallel_dt = 0;
    p->limit = 0.1e6;
    p->threads = 1;
    p->convert_colorspace = 1;
    p->colorspace = 0;
    p->verbose = 1;
    p->populate_nearest = 1;
    p->partition_step = 1;
    p->ndims = 6;
    p->nchroma = 1;
    p->ntables = 1;
    p->populate_exptime = 0;
    p->init_random = 0;
    p->dt_mode = 0;
    p->dt_algo = 1;
    p->dt_iters = -1;
    p->query_step = 1;
    p->run_dt = 1;
    p->do_prop = 1;
    p->do_rs = 1;
    p->allowed_index = 1;
    p->spatial = 0;
    p->patch_w = 8;
    p->kcoherence_step = 1;
    p->coherence_spatial = 0.0;
    p->coherence_temporal = 0.0;
    p->table_ratio = 2.0;
    p->recalc_dist_temporal = 1;
    p->is_descriptor = 0;
    p->descriptor_padded = 0;
    p->lookup_algo = 0;
    p->flann_build_step = 1;
    p->flann_reset_step = 10;
    p->query_iters = 2;
    p->prop_iters = 0;
    p->kcoherence = 0;
    p->kcoherence_min_dist = 2;
    p->kcoherence_algo = 0;
    p->dim_algo = 0;
    p->populate_random = 1;
    p->kcoherence_iter = -1;
    p->grid_ndims = -1;
    p->prop_dist = 0;
    p->incoherence = 0;
    p->triangle_factor = 2.0;
    p->pca_samples = 1000;
    p->pca_mean = 0;
    p->pca_subtract_mean = 1;
    p->sanitize_input = 1;
    p->do_table_lookup = 1;
    p->gpu_prop_passes = 0;
    p->gpu_jump = 0;
    p->gpu_pull_max = 0;
    p->gpu_tile = 0;
    p->gpu_kc_max = 0;
    pt_params_set_speed(p, 3);
}

pt_status pt_params_set_speed(pt_params *p, int speed) {
    if (!p) return pt_fail(PT_BAD_ARG, "null params");
    if (speed < 0 || speed > 9) return pt_fail(PT_BAD_ARG, "set_speed(i), i=%d, expected integer in 0...9", speed);
    return apply_string(p, SPEED_PRESETS[speed]);
}

pt_status pt_params_from_switches(pt_params *p, const char *switches) {
    if (!p || !switches) return pt_fail(PT_BAD_ARG, "null argument");
    return apply_string(p, std::string(switches));
}

}  // extern "C"
