// cudaamica: command-line drop-in for the reference's `cudaamica -f <params>`
// (src/cudaamica.cu:17-43), driving the engine through its C ABI.
//
// Reference keys are read in the reference's order with the reference's
// matching rules (src/params.c, src/config.c:12-213), because those rules are
// part of what an existing params file means:
//   - a line whose first character is '#' is skipped;
//   - a key is looked up by scanning the lines for the first one that CONTAINS
//     it; that line is cut at its first space even when its first word is a
//     different key, and the scan goes on (so an earlier lookup can hide a
//     later key that shares its line);
//   - the value is the second space-separated word; integers and reals are
//     read with atol/atof (a trailing newline is ignored), strings lose their
//     last character (the newline), booleans are on / off / none (1 / 0 / 2);
//   - a missing update_rho leaves rho fixed and sets do_newton to 1
//     (src/config.c:146-153).
// The reference crashes on a '#' line for every non-string key; here such a
// line is simply a comment.
//
// Extension keys (not in the reference) are read afterwards by exact first
// word, without the quirks: precision (mixed | fp32), do_reject (on/off),
// rejsig, rejstart, rejint, maxrej, phi_split (split correction of phi in the
// mixed form: 0 never, 1 always, 2 automatic) and phi_split_rel (its
// threshold), tc_shape (tile shape of the fused E-step: 0, 1 or 2),
// ainitfile / cinitfile (raw float32, one n x n column-major block
// / n values per model, the last block repeated for the remaining models),
// lrate, lratemax, lnatrate, lratefact, rho0, rholrate, rhomin, rhomax,
// maxdec, seed.
//
// Output: the reference's raw FP64 files (amica_write_outputs) and its stdout
// lines "Iteration %lu: lrate %.16f LL %.16f ", "Likelihood decreasing!" and
// "Iteration %lu times = %lu ticks, %lu ms ".  llfile holds the LL of every
// iteration, 1..maxiter (the reference writes an unset value first and drops
// the last iteration, src/amica.cu:800,2806-2813).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "amica_b200.h"

namespace {

// ------------------------------------------------------------ params file
struct Lines {
    std::vector<std::string> raw;     // as read, for the extension keys
    std::vector<std::vector<char>> q; // mutable copies, for the reference keys
    std::vector<bool> present;        // false for '#' lines
};

bool read_lines(const char* path, Lines* L) {
    FILE* f = fopen(path, "r");
    if (!f) return false;
    std::vector<char> buf(5000);
    while (fgets(buf.data(), (int)buf.size(), f)) {
        std::string s(buf.data());
        L->raw.push_back(s);
        L->present.push_back(!s.empty() && s[0] != '#');
        std::vector<char> v(s.begin(), s.end());
        v.push_back('\0');
        L->q.push_back(v);
    }
    fclose(f);
    return true;
}

// The reference's lookup: first line containing `key`; cut it at the first
// space-run (strtok semantics); if its first word is `key`, return the second
// word (up to the next space) or nullptr with *bad = true when there is none.
const char* ref_lookup(Lines* L, const char* key, bool* found, bool* bad) {
    *found = false;
    *bad = false;
    for (size_t i = 0; i < L->q.size(); i++) {
        if (!L->present[i]) continue;
        char* line = L->q[i].data();
        if (!strstr(line, key)) continue;
        // strtok(line, " "): skip leading spaces, cut after the first word
        char* p = line;
        while (*p == ' ') p++;
        if (*p == '\0') { *found = true; *bad = true; return nullptr; }
        char* w = p;
        while (*p && *p != ' ') p++;
        char* rest = nullptr;
        if (*p) { *p = '\0'; rest = p + 1; }
        if (strcmp(w, key) == 0) {
            *found = true;
            if (!rest) { *bad = true; return nullptr; }
            while (*rest == ' ') rest++;
            if (*rest == '\0') { *bad = true; return nullptr; }
            char* e = rest;
            while (*e && *e != ' ') e++;
            *e = '\0';
            return rest;
        }
        // another key's line: left cut, scan on
    }
    return nullptr;
}

// status: 0 found, AMICA_ERR_NOPARAM missing, AMICA_ERR_INVALIDPARAM malformed
int ref_long(Lines* L, const char* key, int64_t* out) {
    bool found, bad;
    const char* v = ref_lookup(L, key, &found, &bad);
    if (!found) return AMICA_ERR_NOPARAM;
    if (bad) return AMICA_ERR_INVALIDPARAM;
    *out = atol(v);
    return AMICA_OK;
}
int ref_bool(Lines* L, const char* key, int64_t* out) {
    bool found, bad;
    const char* v = ref_lookup(L, key, &found, &bad);
    if (!found) return AMICA_ERR_NOPARAM;
    if (bad) return AMICA_ERR_INVALIDPARAM;
    std::string s(v);
    if (!s.empty() && s.back() == '\n') s.pop_back();
    if (s == "on") *out = 1;
    else if (s == "off") *out = 0;
    else if (s == "none") *out = 2;
    else return AMICA_ERR_INVALIDPARAM;
    return AMICA_OK;
}
int ref_string(Lines* L, const char* key, std::string* out) {
    bool found, bad;
    const char* v = ref_lookup(L, key, &found, &bad);
    if (!found) return AMICA_ERR_NOPARAM;
    if (bad) return AMICA_ERR_INVALIDPARAM;
    std::string s(v);
    if (!s.empty()) s.pop_back();            // the reference drops the last character
    *out = s;
    return AMICA_OK;
}
int ref_long_list(Lines* L, const char* key, std::vector<int64_t>* out) {
    for (size_t i = 0; i < L->q.size(); i++) {
        if (!L->present[i]) continue;
        char* line = L->q[i].data();
        if (!strstr(line, key)) continue;
        char* save = nullptr;
        char* w = strtok_r(line, " ", &save);
        if (!w) return AMICA_ERR_INVALIDPARAM;
        if (strcmp(w, key) != 0) continue;
        out->clear();
        while ((w = strtok_r(nullptr, " ", &save)) != nullptr) out->push_back(atol(w));
        return AMICA_OK;
    }
    return AMICA_ERR_NOPARAM;
}

// Extension keys: exact first word on the unmodified line.
bool ext_value(const Lines& L, const char* key, std::string* out) {
    for (size_t i = 0; i < L.raw.size(); i++) {
        if (!L.present[i]) continue;
        char tmp[5000];
        snprintf(tmp, sizeof(tmp), "%s", L.raw[i].c_str());
        char* save = nullptr;
        char* w = strtok_r(tmp, " \t\r\n", &save);
        if (!w || strcmp(w, key) != 0) continue;
        char* v = strtok_r(nullptr, " \t\r\n", &save);
        *out = v ? v : "";
        return true;
    }
    return false;
}

// ------------------------------------------------------------ file helpers
bool read_floats(const std::string& path, std::vector<float>* v, size_t count) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return false;
    v->resize(count);
    const size_t got = fread(v->data(), sizeof(float), count, f);
    fclose(f);
    return got == count;
}

// per-model blocks of `block` floats; missing trailing models repeat the last block
bool read_init(const std::string& path, size_t block, int64_t M, std::vector<double>* out) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return false;
    std::vector<float> all;
    std::vector<float> buf(block);
    while (fread(buf.data(), sizeof(float), block, f) == block && (int64_t)(all.size() / block) < M)
        all.insert(all.end(), buf.begin(), buf.end());
    fclose(f);
    if (all.empty()) return false;
    const std::vector<float> last(all.end() - block, all.end());
    while ((int64_t)(all.size() / block) < M) all.insert(all.end(), last.begin(), last.end());
    out->assign(all.begin(), all.begin() + block * M);
    return true;
}

void usage() {
    printf("\nUsage: cudaamica -f <params file>\n\n");
}

}  // namespace

int main(int argc, char** argv) {
    const char* params = nullptr;
    for (int i = 1; i + 1 < argc; i++)
        if (strcmp(argv[i], "-f") == 0) params = argv[i + 1];
    if (!params) {
        printf("\nERROR::Script configuration file is mandatory\n\n\n");
        usage();
        return AMICA_ERR_NOFILE;
    }
    Lines L;
    printf("Opening config file %s\n", params);
    if (!read_lines(params, &L)) {
        fprintf(stderr, "ERROR: cannot open %s\n", params);
        return AMICA_ERR_INVALIDCONFIG;
    }
    amica_cfg cfg;
    amica_default_cfg(&cfg);
    cfg.update_rho = 0;                 // the reference's global starts at zero
    int status = AMICA_OK;
    auto fail = [&](int rc, const char* what) {
        fprintf(stderr, "ERROR: Invalid %s\n", what);
        status = rc;
    };
    std::vector<int64_t> devs;
    int rc = ref_long_list(&L, "devices", &devs);
    if (rc == AMICA_OK && !devs.empty()) cfg.device = devs[0];
    else if (rc != AMICA_ERR_NOPARAM && rc != AMICA_OK) fail(rc, "devices specification (devices)");
    std::string datafile, spherefile;
    if ((rc = ref_string(&L, "datafile", &datafile)) != AMICA_OK) fail(rc, "data file (datafile)");
    if ((rc = ref_long(&L, "nchannels", &cfg.nchannels)) != AMICA_OK) fail(rc, "number of channels (nchannels)");
    if ((rc = ref_long(&L, "nsamples", &cfg.nsamples)) != AMICA_OK) fail(rc, "number of samples (nsamples)");
    auto opt_long = [&](const char* key, int64_t* dst, const char* what) {
        const int r = ref_long(&L, key, dst);
        if (r != AMICA_OK && r != AMICA_ERR_NOPARAM) fail(r, what);
    };
    auto opt_bool = [&](const char* key, int64_t* dst, const char* what) {
        const int r = ref_bool(&L, key, dst);
        if (r != AMICA_OK && r != AMICA_ERR_NOPARAM) fail(r, what);
    };
    opt_long("do_sphere", &cfg.do_sphere, "sphering value (do_sphere)");
    opt_long("maxiter", &cfg.maxiter, "number of maximum iterations (maxiter)");
    opt_long("nsdm", &cfg.nsdm, "number of source density models (nsdm)");
    opt_long("nmmodels", &cfg.nmmodels, "number of ICA mixture models (nmmodels)");
    if ((rc = ref_string(&L, "spherefile", &spherefile)) != AMICA_OK) fail(rc, "sphere file (spherefile)");
    opt_long("block_size", &cfg.block_size, "block size (block_size)");
    opt_bool("fix_init", &cfg.fix_init, "fix_init value (fix_init)");
    const char* file_keys[] = {"afile", "weightsfile", "khindsfile", "cfile", "llfile", "ltallfile",
                               "gmfile", "alphafile", "mufile", "betafile", "rhofile"};
    std::string files[11];
    bool have_file[11] = {};
    for (int k = 0; k < 11; k++) {
        const int r = ref_string(&L, file_keys[k], &files[k]);
        if (r == AMICA_OK) have_file[k] = true;
        else if (r != AMICA_ERR_NOPARAM) fail(r, file_keys[k]);
    }
    opt_bool("do_newton", &cfg.do_newton, "update policy (doNewton)");
    rc = ref_long(&L, "update_rho", &cfg.update_rho);
    if (rc == AMICA_ERR_NOPARAM) cfg.do_newton = 1;          // src/config.c:146-153
    else if (rc != AMICA_OK) fail(rc, "rho update policy (update_rho)");
    opt_long("rho_start_iter", &cfg.rho_start_iter, "number of iterations to update rho (rho_start_iter)");
    opt_long("newt_start_iter", &cfg.newt_start_iter, "number of iterations to do newton (newt_start_iter)");

    // extension keys
    std::string v;
    if (ext_value(L, "precision", &v)) {
        if (v == "mixed") cfg.precision = AMICA_PREC_MIXED;
        else if (v == "fp32") cfg.precision = AMICA_PREC_FP32;
        else fail(AMICA_ERR_INVALIDPARAM, "precision (mixed | fp32)");
    }
    if (ext_value(L, "do_reject", &v)) {
        if (v == "on" || v == "1") cfg.do_reject = 1;
        else if (v == "off" || v == "0") cfg.do_reject = 0;
        else fail(AMICA_ERR_INVALIDPARAM, "do_reject (on | off)");
    }
    struct { const char* k; int64_t* p; } ints[] = {{"rejstart", &cfg.rejstart}, {"rejint", &cfg.rejint},
                                                   {"maxrej", &cfg.maxrej}, {"maxdec", &cfg.maxdec},
                                                   {"seed", &cfg.seed}, {"phi_split", &cfg.phi_split},
                                                   {"tc_shape", &cfg.tc_shape}};
    for (auto& e : ints)
        if (ext_value(L, e.k, &v)) *e.p = atol(v.c_str());
    struct { const char* k; double* p; } reals[] = {{"rejsig", &cfg.rejsig}, {"lrate", &cfg.lrate0},
                                                   {"lratemax", &cfg.lratemax}, {"lnatrate", &cfg.lnatrate},
                                                   {"lratefact", &cfg.lratefact}, {"rho0", &cfg.rho0},
                                                   {"rholrate", &cfg.rholrate}, {"rhomin", &cfg.rhomin},
                                                   {"rhomax", &cfg.rhomax}, {"phi_split_rel", &cfg.phi_split_rel}};
    for (auto& e : reals)
        if (ext_value(L, e.k, &v)) *e.p = atof(v.c_str());
    std::string ainit, cinit;
    const bool have_ainit = ext_value(L, "ainitfile", &ainit);
    const bool have_cinit = ext_value(L, "cinitfile", &cinit);
    if (status != AMICA_OK) return status;

    printf("datafile %s\nnchannels %ld\nnsamples %ld\nnmmodels %ld\nnsdm %ld\nmaxiter %ld\n"
           "do_sphere %ld\ndo_newton %ld\nupdate_rho %ld\nnewt_start_iter %ld\nrho_start_iter %ld\n"
           "precision %s\ndo_reject %ld\n",
           datafile.c_str(), (long)cfg.nchannels, (long)cfg.nsamples, (long)cfg.nmmodels,
           (long)cfg.nsdm, (long)cfg.maxiter, (long)cfg.do_sphere, (long)cfg.do_newton,
           (long)cfg.update_rho, (long)cfg.newt_start_iter, (long)cfg.rho_start_iter,
           cfg.precision == AMICA_PREC_MIXED ? "mixed" : "fp32", (long)cfg.do_reject);

    const int64_t n = cfg.nchannels, T = cfg.nsamples, M = cfg.nmmodels;
    std::vector<float> x;
    if (!read_floats(datafile, &x, (size_t)n * T)) {
        fprintf(stderr, "ERROR: cannot read %ld x %ld float32 values from %s\n", (long)T, (long)n,
                datafile.c_str());
        return AMICA_ERR_NOFILE;
    }
    std::vector<double> A0, c0;
    if (have_ainit && !read_init(ainit, (size_t)n * n, M, &A0)) return AMICA_ERR_NOFILE;
    if (have_cinit && !read_init(cinit, (size_t)n, M, &c0)) return AMICA_ERR_NOFILE;

    cfg.verbose = 0;                    // the per-iteration lines are printed below
    amica_ctx* ctx = nullptr;
    rc = amica_create(&cfg, &ctx);
    if (rc != AMICA_OK) {
        fprintf(stderr, "ERROR: %s\n", amica_status_string(rc));
        return rc;
    }
    rc = amica_load_data(ctx, x.data(), n, T);
    if (rc == AMICA_OK) rc = amica_preprocess(ctx);
    if (rc == AMICA_OK) rc = amica_init(ctx, have_ainit ? A0.data() : nullptr, have_cinit ? c0.data() : nullptr);
    std::vector<amica_iter_out> hist(cfg.maxiter > 0 ? cfg.maxiter : 1);
    int64_t done = 0;
    while (rc == AMICA_OK && done < cfg.maxiter) {
        const int64_t k = cfg.maxiter - done < 100 ? cfg.maxiter - done : 100;
        rc = amica_run(ctx, k, hist.data() + done);
        for (int64_t i = 0; i < k && rc == AMICA_OK; i++) {
            // src/amica.cu:1983-1986, :2540 (ticks here are microseconds of device time)
            const amica_iter_out& o = hist[done + i];
            printf("Iteration %lu: lrate %.16f LL %.16f \n", (unsigned long)o.iter, o.lrate, o.ll);
            if (o.ll_decreased) printf("Likelihood decreasing!\n");
            if (o.nrejected) printf("Rejected %ld samples\n", (long)o.nrejected);
            printf("Iteration %lu times = %lu ticks, %lu ms \n", (unsigned long)o.iter,
                   (unsigned long)llround(o.device_ms * 1000.0), (unsigned long)llround(o.device_ms));
        }
        done += k;
    }
    if (rc == AMICA_OK) {
        amica_paths p;
        memset(&p, 0, sizeof(p));
        const char** slots[] = {&p.afile, &p.weightsfile, nullptr, &p.cfile, &p.llfile, &p.ltallfile,
                                &p.gmfile, &p.alphafile, &p.mufile, &p.betafile, &p.rhofile};
        for (int k = 0; k < 11; k++)
            if (slots[k] && have_file[k]) *slots[k] = files[k].c_str();
        p.spherefile = spherefile.c_str();
        rc = amica_write_outputs(ctx, &p);
    }
    if (rc != AMICA_OK) fprintf(stderr, "ERROR: %s\n", amica_status_string(rc));
    amica_destroy(ctx);
    return rc;
}
