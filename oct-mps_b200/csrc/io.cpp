// Input parsers and output writers in the reference's file formats.
//
// .opt  : read_simulation_data, src/octmps_io.cpp:504-645
// .mci  : Bias_Read, src/bias.cpp:9-110
// output: Write_Bias_Parameters and WriteResult, src/octmps_io.cpp:237-437
//
// The line readers keep the reference's rules (src/octmps_io.cpp:444-494):
// a data line is the next line from which sscanf converts at least one
// number; lines with more numbers than asked are an error; the buffer sizes
// (200 characters for numbers, 256 for integers and names) are the same, so
// over-long lines split the same way.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "octmps_host.h"

namespace {

const int kFloatLine = 200;
const int kStrLen = 256;

struct LineReader {
    FILE *f;
    // Next data line parsed with `fmt` into up to 5 values.  Returns the
    // count converted (>0), or 0 on end of file / too many values.
    template <typename V>
    int read(const char *fmt, int want, V *out, int bufsize) {
        char line[kStrLen + 1];
        int ii = 0;
        while (ii <= 0) {
            if (feof(f)) return 0;
            if (!fgets(line, bufsize, f)) return 0;
            V tmp[5] = {0, 0, 0, 0, 0};
            ii = sscanf(line, fmt, &tmp[0], &tmp[1], &tmp[2], &tmp[3], &tmp[4]);
            if (ii > want) return 0;
            if (ii > 0)
                for (int k = 0; k < 5; ++k) out[k] = tmp[k];
        }
        return ii;
    }
    int floats(int n, float *out) { return read("%f %f %f %f %f", n, out, kFloatLine); }
    int doubles(int n, double *out) { return read("%lf %lf %lf %lf %lf", n, out, kFloatLine); }
    int ints(int n, int *out) { return read("%d %d %d %d %d", n, out, kStrLen); }
};

int is_letter(char a) { return (a >= 'A' && a <= 'Z') || (a >= 'a' && a <= 'z'); }

std::string join(const char *dir, const char *name) {
    if (!dir || !*dir) return name;
    std::string s(dir);
    if (s.back() != '/') s += '/';
    return s + name;
}

}  // namespace

extern "C" octmps_status octmps_read_opt(const char *path, octmps_sim *out) {
    if (!path || !out) return OCTMPS_ERR_INVALID_ARG;
    FILE *f = fopen(path, "r");
    if (!f) return OCTMPS_ERR_IO;
    LineReader r{f};
    memset(out, 0, sizeof *out);
    float ft[5];
    int it[5];
    double dt[5];
    octmps_status st = OCTMPS_ERR_IO;
    do {
        if (!r.floats(1, ft)) break;  // file version, ignored
        if (!r.ints(1, it)) break;    // number of runs
        if (it[0] < 1) break;
        // Only run 1 is read: the reference applies the .mci parameters
        // and the probe scan to simulations[0] alone (src/bias.cpp:28-104,
        // src/main.cu:948-959).
        char line[kStrLen + 1], name[kStrLen + 1];
        char aorb = 0;
        int ii = 0;
        bool ok = true;
        while (ii <= 0) {
            if (!fgets(line, kStrLen, f)) { ok = false; break; }
            ii = sscanf(line, "%256s %c", name, &aorb);
            if (feof(f) || ii > 2) { ok = false; break; }
            if (ii > 0) ii = is_letter(name[0]);
        }
        if (!ok) break;
        unsigned int nph = 0;
        ii = 0;
        while (ii <= 0) {
            if (!fgets(line, kStrLen, f)) { ok = false; break; }
            nph = 0;
            ii = sscanf(line, "%u", &nph);
            if (feof(f) || ii > 1) { ok = false; break; }
        }
        if (!ok) break;
        out->number_of_photons = nph;
        if (!r.ints(1, it)) break;
        const int n_regions = it[0] + 1;
        if (n_regions < 2 || n_regions > OCTMPS_MAX_REGIONS) { st = OCTMPS_ERR_INVALID_ARG; break; }
        out->n_regions = n_regions;
        if (!r.doubles(1, dt)) break;
        out->regions[0].n = dt[0];
        for (int k = 1; k < n_regions && ok; ++k) {
            if (!r.doubles(4, dt)) { ok = false; break; }
            out->regions[k].n = dt[0];
            out->regions[k].mua = dt[1];
            out->regions[k].mus = dt[2];
            out->regions[k].g = dt[3];
        }
        if (!ok) break;
        if (!r.doubles(3, dt)) break;
        out->start_x = dt[0];
        out->step_x = dt[1];
        out->end_x = dt[2];
        st = OCTMPS_OK;
    } while (0);
    fclose(f);
    return st;
}

extern "C" octmps_status octmps_read_mci(const char *path, octmps_sim *s) {
    if (!path || !s) return OCTMPS_ERR_INVALID_ARG;
    FILE *f = fopen(path, "r");
    if (!f) return OCTMPS_ERR_IO;
    LineReader r{f};
    float ft[5];
    int it[5];
    octmps_status st = OCTMPS_ERR_IO;
    do {
        if (!r.ints(1, it)) break;
        s->type_simulation = it[0];
        if (!r.ints(1, it)) break;
        s->type_bias = it[0];
        if (!r.floats(1, ft)) break;
        s->backward_bias_coefficient = ft[0];
        if (!r.floats(1, ft)) break;
        s->target_depth_min = ft[0];
        if (!r.floats(1, ft)) break;
        s->target_depth_max = ft[0];
        if (!r.floats(1, ft)) break;
        s->coherence_length_source = ft[0];
        if (!r.ints(1, it)) break;
        s->record_photons_flag = it[0];
        if (!r.floats(1, ft)) break;
        s->max_collecting_radius = ft[0];
        if (!r.floats(1, ft)) break;
        s->max_collecting_angle_deg = ft[0];
        if (!r.floats(1, ft)) break;
        s->probability_additional_bias = ft[0];
        if (!r.floats(1, ft)) break;
        s->max_relative_contribution = ft[0];
        // Derived values, src/bias.cpp:92-104.
        const float kMaxFixedOpticalDepth = 0.12f;
        if (s->target_depth_max < kMaxFixedOpticalDepth)
            s->max_filtered_optical_depth = kMaxFixedOpticalDepth;
        else
            s->max_filtered_optical_depth = s->target_depth_max;
        const double steps = 6 * s->max_filtered_optical_depth / s->coherence_length_source;
        if (!(steps >= 1.0) || steps >= 2147483647.0) { st = OCTMPS_ERR_INVALID_ARG; break; }
        s->num_optical_depth_length_steps = (int32_t)steps;
        s->optical_depth_shift = fmod(s->target_depth_min, s->coherence_length_source);
        s->rnd_step_size_in_tissue = 0.0;
        st = OCTMPS_OK;
    } while (0);
    fclose(f);
    return st;
}

// WriteReflectanceClassI_and_ClassII and its filtered variant
// (src/octmps_io.cpp:302-420): one line per depth bin, "%G,%G,%G,%G,%llu".
static void write_scatt(FILE *f1, FILE *f2, const octmps_sim *s, double probe_x, const double *sum1,
                        const double *sumsq1, const double *sum2, const double *sumsq2,
                        const uint64_t *c1, const uint64_t *c2) {
    const unsigned int n = s->number_of_photons;
    for (long int i = 0; i < s->num_optical_depth_length_steps; i++) {
        double mean1 = sum1[i] / n;
        double var1 = (sumsq1[i] / n - mean1 * mean1) / (n - 1);
        double mean2 = sum2[i] / n;
        double var2 = (sumsq2[i] / n - mean2 * mean2) / (n - 1);
        double depth = i * s->coherence_length_source / 6 + s->optical_depth_shift;
        fprintf(f1, "%G,%G,%G,%G,%llu\n", probe_x, depth, mean1, sqrt(var1),
                (unsigned long long)c1[i]);
        fprintf(f2, "%G,%G,%G,%G,%llu\n", probe_x, depth, mean2, sqrt(var2),
                (unsigned long long)c2[i]);
    }
}

extern "C" octmps_status octmps_write_result(const char *dir, const octmps_sim *s, double probe_x,
                                             const octmps_tally *t) {
    if (!s || !t) return OCTMPS_ERR_INVALID_ARG;
    const int nb = s->num_optical_depth_length_steps;
    // Write_Bias_Parameters (src/octmps_io.cpp:237-300).  It creates
    // FilteredPhotons.mco empty; with RecordPhotonsFlag the file holds the
    // detected-packet records instead (octmps_write_filtered_photons appends
    // them), so it is left alone here.
    if (!(short)s->record_photons_flag) {
        FILE *fp = fopen(join(dir, "FilteredPhotons.mco").c_str(), "w");
        if (fp) fclose(fp);
    }
    FILE *b = fopen(join(dir, "BiasParam.mco").c_str(), "w");
    if (!b) return OCTMPS_ERR_IO;
    fprintf(b, "%llu\t\t\t\t\t# Number of filtered photons\n", (unsigned long long)t->num_filtered);
    fprintf(b, "%llu\t\t\t\t\t# Number of Class I filtered photons\n",
            (unsigned long long)t->num_filtered_class1);
    fprintf(b, "%llu\t\t\t\t\t# Number of Class II filtered photons\n",
            (unsigned long long)t->num_filtered_class2);
    if ((short)s->record_photons_flag) {
        fprintf(b, "\n\n\n\n");
        fprintf(b, "Description of fields in file FilteredPhotons.mco\n\n");
        fprintf(b, "================================================================\n");
        fprintf(b, "Weight | LikelihoodRatio | Radius | AngleRad | OpticalPath | MaxDepth");
    }
    fprintf(b, "%hd\t\t\t\t\t# Type of simulation\n", (short)s->type_simulation);
    fprintf(b, "%hd\t\t\t\t\t# Type of bias\n", (short)s->type_bias);
    fprintf(b, "%u\t\t\t\t\t# Number of photon packets\n", s->number_of_photons);
    fprintf(b, "%G\t\t\t\t\t# Backward bias coefficient\n", s->backward_bias_coefficient);
    fprintf(b, "%G\t\t\t\t\t# Target depth min [cm]\n", s->target_depth_min);
    fprintf(b, "%G\t\t\t\t\t# Target depth max [cm]\n", s->target_depth_max);
    fprintf(b, "%G\t\t\t\t\t# Coherence length source [cm]\n", s->coherence_length_source);
    fprintf(b, "%G\t\t\t\t\t# Max collecting radius [cm]\n", s->max_collecting_radius);
    fprintf(b, "%G\t\t\t\t\t# Max collecting angle [grad]\n", s->max_collecting_angle_deg);
    fprintf(b, "%hd\t\t\t\t\t# Record photons flag\n", (short)s->record_photons_flag);
    fprintf(b, "%G\t\t\t\t\t# Probability of additional bias\n", s->probability_additional_bias);
    fprintf(b, "%G\t\t\t\t\t# Maximum relative contribution to bin per post-processed sample\n",
            s->max_relative_contribution);
    fclose(b);

    // WriteResult (src/octmps_io.cpp:422-437): unfiltered, then filtered.
    FILE *f1 = fopen(join(dir, "ClassI_Scatt.out").c_str(), "a");
    FILE *f2 = fopen(join(dir, "ClassII_Scatt.out").c_str(), "a");
    if (!f1 || !f2) {
        if (f1) fclose(f1);
        if (f2) fclose(f2);
        return OCTMPS_ERR_IO;
    }
    write_scatt(f1, f2, s, probe_x, t->sum1, t->sumsq1, t->sum2, t->sumsq2, t->count1, t->count2);
    fclose(f1);
    fclose(f2);

    // Filtered: drop the largest single contribution of a bin when it
    // exceeds the allowed fraction of the bin's sum (src/octmps_io.cpp:361-375).
    double *fs1 = new double[nb], *fq1 = new double[nb], *fs2 = new double[nb], *fq2 = new double[nb];
    for (int i = 0; i < nb; ++i) {
        fs1[i] = t->sum1[i];
        fq1[i] = t->sumsq1[i];
        fs2[i] = t->sum2[i];
        fq2[i] = t->sumsq2[i];
        if (t->max1[i] > s->max_relative_contribution * fs1[i]) {
            fs1[i] -= t->max1[i];
            fq1[i] -= t->max1[i] * t->max1[i];
        }
        if (t->max2[i] > s->max_relative_contribution * fs2[i]) {
            fs2[i] -= t->max2[i];
            fq2[i] -= t->max2[i] * t->max2[i];
        }
    }
    f1 = fopen(join(dir, "ClassI_ScattFilt.out").c_str(), "a");
    f2 = fopen(join(dir, "ClassII_ScattFilt.out").c_str(), "a");
    octmps_status st = OCTMPS_OK;
    if (!f1 || !f2) st = OCTMPS_ERR_IO;
    else write_scatt(f1, f2, s, probe_x, fs1, fq1, fs2, fq2, t->count1, t->count2);
    if (f1) fclose(f1);
    if (f2) fclose(f2);
    delete[] fs1;
    delete[] fq1;
    delete[] fs2;
    delete[] fq2;
    return st;
}

extern "C" int64_t octmps_safeprimes_read(const char *path, uint32_t *out, uint64_t max_count) {
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    uint64_t n = 0;
    unsigned int a, t1, t2;
    while (n < max_count && fscanf(f, "%u %u %u", &a, &t1, &t2) == 3) out[n++] = a;
    fclose(f);
    return (int64_t)n;
}

// FilteredPhotons.mco records (RecordPhotonsFlag): the fields BiasParam.mco
// lists for the file (src/octmps_io.cpp:259-270), after the A-scan's probe
// position; the angle is acos of the stored cosine.
extern "C" octmps_status octmps_write_filtered_photons(const char *dir, double probe_x,
                                                       const octmps_photon_record *r, uint64_t n) {
    if (n && !r) return OCTMPS_ERR_INVALID_ARG;
    FILE *f = fopen(join(dir, "FilteredPhotons.mco").c_str(), "a");
    if (!f) return OCTMPS_ERR_IO;
    for (uint64_t i = 0; i < n; ++i)
        fprintf(f, "%G\t%G\t%G\t%G\t%G\t%G\t%G\n", probe_x, r[i].weight, r[i].likelihood,
                r[i].radius, acos(r[i].cos_angle), r[i].optical_path, r[i].max_depth);
    return fclose(f) == 0 ? OCTMPS_OK : OCTMPS_ERR_IO;
}
