/*
 * FP64 CPU oracle for the pripps Debye path.
 *
 * TEST INFRASTRUCTURE ONLY. The parity tests and the CPU-baseline leg of
 * bench.py compare the backend against this file; no product code path links,
 * loads or calls it. It restates, loop for loop, the reference's f64 Debye
 * code so that results can be compared on identical inputs:
 *
 *   sinc                  src/debye.rs:17-24
 *   self_intensity_at_q   src/debye.rs:214-232
 *   cross_intensity_at_q  src/debye.rs:236-250
 *   build_model (per q)   src/debye.rs:90-130  (3 self sums + 3 cross sums)
 *   intensity_at_q        src/debye.rs:200-211 (vacuum)
 *   DebyeTerms::combine   src/debye.rs:187-194
 *   linear_q_values       src/q_sampler.rs:24-29
 *   eval_gaussian         src/formfactor.rs:368-375
 *   eval_polynomium       src/formfactor.rs:378-385
 *   interpolate           src/formfactor.rs:388-408
 *   united table          src/formfactor.rs:669-682
 *   fraser_form_factor    src/solvent/fraser.rs:48-57 (+ SingleGaussian eval
 *                         src/formfactor.rs:196)
 *   SASA shell weight     src/solvent/sasa.rs:54-59
 *   Direct transform rows  src/explicit.rs:138-147 (complex_amplitude),
 *                         :208-230 (vacuum_rows: per-molecule F_m, |Σ F_m|²,
 *                         Σ |F_m|²)
 *   build_model with dummies at their own positions (grid / Voronoi /
 *   caller-supplied DummySets): src/debye.rs:83-130 with
 *   DummySet::form_factors_at src/solvent/mod.rs:357-374
 *
 * Build with -ffp-contract=off: the reference (Rust) never contracts a*b+c
 * into an FMA except where it calls mul_add explicitly, which is restated here
 * with fma(). sin/exp/sqrt come from the host libm, the same functions the
 * reference's f64 methods call on Linux.
 *
 * The per-q loop is parallel over q with a pthread pool pulling q indices
 * from a shared counter, the way the reference uses rayon's par_iter over q
 * (src/debye.rs:90-92, src/q_sampler.rs:75-79).
 */
#include <math.h>
#include <pthread.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <unistd.h>

/* src/debye.rs:17-24 */
double pdo_sinc(double x) {
    const double NEARLY_ZERO = 1e-8;
    if (fabs(x) < NEARLY_ZERO) return 1.0;
    return sin(x) / x;
}

/* src/q_sampler.rs:24-29: inclusive endpoints, (nq-1).max(1) denominator. */
void pdo_linear_q_values(double qmin, double qmax, size_t nq, double *out) {
    double denom = (double)(nq > 1 ? nq - 1 : 1);
    for (size_t i = 0; i < nq; ++i) out[i] = qmin + (qmax - qmin) * (double)i / denom;
}

/* nalgebra Vector3::norm: sqrt of the sum of squares. */
static inline double dist3(const double *a, const double *b) {
    double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return sqrt(dx * dx + dy * dy + dz * dz);
}

/* Compensated variants: the same sums with the running accumulators in long
 * double (64-bit mantissa on x86-64), used to tell the oracle's own rounding
 * from a kernel's error when a comparison sits at the 1e-10 level. */
static double self_intensity_ld(const double *xyz, const double *f, size_t n, double q) {
    long double diagonal = 0.0L;
    for (size_t i = 0; i < n; ++i) diagonal += (long double)f[i] * f[i];
    if (n < 2) return (double)diagonal;
    long double off = 0.0L;
    for (size_t i = 0; i + 1 < n; ++i) {
        const double *pi = xyz + 3 * i;
        for (size_t j = i + 1; j < n; ++j) {
            double r = dist3(pi, xyz + 3 * j);
            off += (long double)(f[i] * f[j]) * pdo_sinc(q * r);
        }
    }
    return (double)(2.0L * off + diagonal);
}

static double cross_intensity_ld(const double *axyz, const double *af, size_t na,
                                 const double *bxyz, const double *bf, size_t nb, double q) {
    long double total = 0.0L;
    for (size_t a = 0; a < na; ++a)
        for (size_t b = 0; b < nb; ++b)
            total += (long double)(af[a] * bf[b]) * pdo_sinc(q * dist3(axyz + 3 * a, bxyz + 3 * b));
    return (double)total;
}

/* src/debye.rs:214-232: diagonal Σf² first, then i<j (ascending j), then
 * 2.0.mul_add(off, diag). */
double pdo_self_intensity(const double *xyz, const double *f, size_t n, double q) {
    double diagonal = 0.0;
    for (size_t i = 0; i < n; ++i) diagonal += f[i] * f[i];
    if (n < 2) return diagonal;
    double off = 0.0;
    for (size_t i = 0; i + 1 < n; ++i) {
        double fi = f[i];
        const double *pi = xyz + 3 * i;
        for (size_t j = i + 1; j < n; ++j) {
            double r = dist3(pi, xyz + 3 * j);
            off += fi * f[j] * pdo_sinc(q * r);
        }
    }
    return fma(2.0, off, diagonal);
}

/* src/debye.rs:236-250: every (a, b) pair, coincident points included. */
double pdo_cross_intensity(const double *axyz, const double *af, size_t na,
                           const double *bxyz, const double *bf, size_t nb, double q) {
    double total = 0.0;
    for (size_t a = 0; a < na; ++a) {
        const double *pa = axyz + 3 * a;
        double fa = af[a];
        for (size_t b = 0; b < nb; ++b) {
            total += fa * bf[b] * pdo_sinc(q * dist3(pa, bxyz + 3 * b));
        }
    }
    return total;
}

/* src/debye.rs:187-194 */
double pdo_combine(const double *t6, double volume_scale, double contrast_density) {
    return t6[0] + volume_scale * volume_scale * t6[1] +
           contrast_density * contrast_density * t6[2] - 2.0 * volume_scale * t6[3] +
           2.0 * contrast_density * t6[4] - 2.0 * volume_scale * contrast_density * t6[5];
}

/* ---- q-parallel loop (rayon par_iter stand-in) ---- */

typedef struct {
    size_t n;
    const double *xyz;
    const uint32_t *species;
    const double *ff_atoms, *ff_excluded, *hyd_weights, *ff_water;
    /* Dummy sets at their own positions (sets = 1): n_exc excluded dummies at
     * exc_xyz with form factor row exc_kind[i] of ff_excluded; n_hyd hydration
     * dummies at hyd_xyz, B_i = hyd_weights[i]·ff_water. With sets = 0 both
     * sets sit at the atoms (exc_kind = species). */
    int sets;
    size_t n_exc, n_hyd;
    const double *exc_xyz, *hyd_xyz;
    const uint32_t *exc_kind;
    const double *qv;
    size_t nq;
    const uint32_t *q_index;
    size_t nqi;
    int solvent; /* 0: vacuum (out[t]), 1: six terms (out[6t..6t+5]) */
    int precise; /* 1: long double accumulators */
    double *out;
    size_t next; /* shared work counter */
    pthread_mutex_t lock;
    int failed;
} pdo_job;

static long pdo_take(pdo_job *jb) {
    long t = -1;
    pthread_mutex_lock(&jb->lock);
    if (jb->next < jb->nqi) t = (long)jb->next++;
    pthread_mutex_unlock(&jb->lock);
    return t;
}

static void *pdo_worker(void *arg) {
    pdo_job *jb = (pdo_job *)arg;
    size_t n = jb->n;
    size_t n_exc = jb->sets ? jb->n_exc : (jb->ff_excluded ? n : 0);
    size_t n_hyd = jb->sets ? jb->n_hyd : (jb->hyd_weights ? n : 0);
    const double *exc_xyz = jb->sets ? jb->exc_xyz : jb->xyz;
    const double *hyd_xyz = jb->sets ? jb->hyd_xyz : jb->xyz;
    const uint32_t *exc_kind = jb->sets ? jb->exc_kind : jb->species;
    double *fa = (double *)malloc(sizeof(double) * (n ? n : 1));
    double *fc = (double *)malloc(sizeof(double) * (n_exc ? n_exc : 1));
    double *fb = (double *)malloc(sizeof(double) * (n_hyd ? n_hyd : 1));
    if (!fa || !fc || !fb) {
        pthread_mutex_lock(&jb->lock);
        jb->failed = 1;
        pthread_mutex_unlock(&jb->lock);
    } else {
        long t;
        while ((t = pdo_take(jb)) >= 0) {
            size_t k = jb->q_index ? jb->q_index[t] : (size_t)t;
            double q = jb->qv[k];
            /* formfactor_by_index (src/formfactor.rs:528-544) */
            for (size_t i = 0; i < n; ++i) fa[i] = jb->ff_atoms[(size_t)jb->species[i] * jb->nq + k];
            double (*selfs)(const double *, const double *, size_t, double) =
                jb->precise ? self_intensity_ld : pdo_self_intensity;
            double (*cross)(const double *, const double *, size_t, const double *,
                            const double *, size_t, double) =
                jb->precise ? cross_intensity_ld : pdo_cross_intensity;
            if (!jb->solvent) {
                jb->out[t] = selfs(jb->xyz, fa, n, q);
                continue;
            }
            /* DummySet::form_factors_at (src/solvent/mod.rs:357-374) */
            for (size_t i = 0; i < n_exc; ++i)
                fc[i] = jb->ff_excluded[(size_t)exc_kind[i] * jb->nq + k];
            if (n_hyd) {
                double shared = jb->ff_water[k];
                for (size_t i = 0; i < n_hyd; ++i) fb[i] = jb->hyd_weights[i] * shared;
            }
            double *o = jb->out + 6 * (size_t)t;
            o[0] = selfs(jb->xyz, fa, n, q);
            o[1] = selfs(exc_xyz, fc, n_exc, q);
            o[2] = selfs(hyd_xyz, fb, n_hyd, q);
            o[3] = cross(jb->xyz, fa, n, exc_xyz, fc, n_exc, q);
            o[4] = cross(jb->xyz, fa, n, hyd_xyz, fb, n_hyd, q);
            o[5] = cross(exc_xyz, fc, n_exc, hyd_xyz, fb, n_hyd, q);
        }
    }
    free(fa);
    free(fc);
    free(fb);
    return NULL;
}

static int pdo_run(pdo_job *jb, int n_threads) {
    if (n_threads <= 0) {
        long c = sysconf(_SC_NPROCESSORS_ONLN);
        n_threads = c > 0 ? (int)c : 1;
    }
    if ((size_t)n_threads > jb->nqi) n_threads = jb->nqi ? (int)jb->nqi : 1;
    pthread_mutex_init(&jb->lock, NULL);
    jb->next = 0;
    jb->failed = 0;
    pthread_t *th = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)n_threads);
    if (!th) return -1;
    int started = 0;
    for (int i = 1; i < n_threads; ++i) {
        if (pthread_create(&th[i], NULL, pdo_worker, jb) != 0) break;
        started = i;
    }
    pdo_worker(jb);
    for (int i = 1; i <= started; ++i) pthread_join(th[i], NULL);
    free(th);
    pthread_mutex_destroy(&jb->lock);
    return jb->failed ? -1 : 0;
}

/*
 * build_model over a subset of the q grid (src/debye.rs:78-136).
 *
 * Inputs are the host-side products of the reference's per-q preparation:
 *   ff_atoms    [n_species][nq]  F_s(q_k)         (formfactor_by_index)
 *   ff_excluded [n_species][nq]  C_s(q_k) or NULL (Fraser dummies at the atoms;
 *                                NULL = ExcludedVolume::Disabled, empty set)
 *   hyd_weights [n]              w_i or NULL      (SASA Weighted dummies at the
 *                                atoms; NULL = Hydration::Disabled, empty set)
 *   ff_water    [nq]             F_H2O(q_k)
 * q_index selects which grid points to evaluate (NULL = all, n_q_index = nq);
 * out is [n_q_index][6] in the DebyeTerms field order
 * (atoms, excluded, hydration, atom_excluded, atom_hydration, excluded_hydration).
 * n_threads <= 0 uses every online core; precise != 0 accumulates in long
 * double. Returns 0, or -1 on allocation failure.
 */
int pdo_build_model(size_t n, const double *xyz, const uint32_t *species, size_t n_species,
                    const double *ff_atoms, const double *ff_excluded,
                    const double *hyd_weights, const double *ff_water, double qmin,
                    double qmax, size_t nq, const uint32_t *q_index, size_t n_q_index,
                    int n_threads, int precise, double *out) {
    (void)n_species;
    double *qv = (double *)malloc(sizeof(double) * (nq ? nq : 1));
    if (!qv) return -1;
    pdo_linear_q_values(qmin, qmax, nq, qv);
    pdo_job jb = {0};
    jb.n = n;
    jb.xyz = xyz;
    jb.species = species;
    jb.ff_atoms = ff_atoms;
    jb.ff_excluded = ff_excluded;
    jb.hyd_weights = hyd_weights;
    jb.ff_water = ff_water;
    jb.qv = qv;
    jb.nq = nq;
    jb.q_index = q_index;
    jb.nqi = q_index ? n_q_index : nq;
    jb.solvent = 1;
    jb.precise = precise;
    jb.out = out;
    int rc = pdo_run(&jb, n_threads);
    free(qv);
    return rc;
}

/*
 * build_model with the excluded-volume and hydration dummies at their own
 * positions (src/debye.rs:83-130): the excluded set is n_exc points exc_xyz
 * whose form factor at q_k is ff_excluded[exc_kind[i]][k] (DummySet::PerDummy,
 * or Weighted with weights folded into the rows); the hydration set is n_hyd
 * points hyd_xyz with B_i(q_k) = hyd_weights[i]·ff_water[k] (DummySet::
 * Weighted, src/solvent/mod.rs:365-371). Either set may be empty (n = 0,
 * pointers NULL). Output as pdo_build_model.
 */
int pdo_build_model_sets(size_t n, const double *xyz, const uint32_t *species,
                         const double *ff_atoms, size_t n_exc, const double *exc_xyz,
                         const uint32_t *exc_kind, const double *ff_excluded, size_t n_hyd,
                         const double *hyd_xyz, const double *hyd_weights,
                         const double *ff_water, double qmin, double qmax, size_t nq,
                         const uint32_t *q_index, size_t n_q_index, int n_threads, int precise,
                         double *out) {
    double *qv = (double *)malloc(sizeof(double) * (nq ? nq : 1));
    if (!qv) return -1;
    pdo_linear_q_values(qmin, qmax, nq, qv);
    pdo_job jb = {0};
    jb.n = n;
    jb.xyz = xyz;
    jb.species = species;
    jb.ff_atoms = ff_atoms;
    jb.ff_excluded = ff_excluded;
    jb.hyd_weights = hyd_weights;
    jb.ff_water = ff_water;
    jb.sets = 1;
    jb.n_exc = n_exc;
    jb.n_hyd = n_hyd;
    jb.exc_xyz = exc_xyz;
    jb.hyd_xyz = hyd_xyz;
    jb.exc_kind = exc_kind;
    jb.qv = qv;
    jb.nq = nq;
    jb.q_index = q_index;
    jb.nqi = q_index ? n_q_index : nq;
    jb.solvent = 1;
    jb.precise = precise;
    jb.out = out;
    int rc = pdo_run(&jb, n_threads);
    free(qv);
    return rc;
}

/* Vacuum path: QSampler::run_parallel -> intensity_at_q -> self sum
 * (src/debye.rs:58-60, :200-211). out is [n_q_index]. */
int pdo_vacuum(size_t n, const double *xyz, const uint32_t *species, const double *ff_atoms,
               double qmin, double qmax, size_t nq, const uint32_t *q_index, size_t n_q_index,
               int n_threads, int precise, double *out) {
    double *qv = (double *)malloc(sizeof(double) * (nq ? nq : 1));
    if (!qv) return -1;
    pdo_linear_q_values(qmin, qmax, nq, qv);
    pdo_job jb = {0};
    jb.n = n;
    jb.xyz = xyz;
    jb.species = species;
    jb.ff_atoms = ff_atoms;
    jb.qv = qv;
    jb.nq = nq;
    jb.q_index = q_index;
    jb.nqi = q_index ? n_q_index : nq;
    jb.solvent = 0;
    jb.precise = precise;
    jb.out = out;
    int rc = pdo_run(&jb, n_threads);
    free(qv);
    return rc;
}

/*
 * Direct transform rows (src/explicit.rs:208-230 with complex_amplitude,
 * :138-147): for q-vector v, the box is cut into n_mol contiguous molecules of
 * n/n_mol points; each molecule's amplitude F_m is folded point by point as
 * (re + f·cos(q·r), im + f·sin(q·r)) with q·r = q_x·x + q_y·y + q_z·z (the
 * nalgebra dot order); a = Σ_m F_m, self = Σ_m |F_m|². ff is
 * [n_kinds][n_vec] (each kind at |q_v|). out[v] = (Re a, Im a, |a|², self).
 */
void pdo_direct_rows(size_t n, const double *xyz, const uint32_t *kind, const double *weight,
                     const double *ff, size_t n_vec, const double *qvec, size_t n_mol,
                     double *out) {
    const size_t m = n_mol ? n / n_mol : n;
    for (size_t v = 0; v < n_vec; ++v) {
        const double qx = qvec[3 * v], qy = qvec[3 * v + 1], qz = qvec[3 * v + 2];
        double ar = 0.0, ai = 0.0, self = 0.0;
        for (size_t p0 = 0; p0 < n; p0 += (m ? m : 1)) {
            double re = 0.0, im = 0.0;
            for (size_t p = p0; p < p0 + m && p < n; ++p) {
                /* DummySet::form_factors_at: w·F for weighted sets */
                const double f = weight ? weight[p] * ff[(size_t)kind[p] * n_vec + v]
                                        : ff[(size_t)kind[p] * n_vec + v];
                const double qr = qx * xyz[3 * p] + qy * xyz[3 * p + 1] + qz * xyz[3 * p + 2];
                re = re + f * cos(qr);
                im = im + f * sin(qr);
            }
            ar += re;
            ai += im;
            self += re * re + im * im;
        }
        out[4 * v] = ar;
        out[4 * v + 1] = ai;
        out[4 * v + 2] = ar * ar + ai * ai;
        out[4 * v + 3] = self;
    }
}

/* ---- form factors (host-side inputs of the path) ---- */

/* src/formfactor.rs:368-375: s² = q²/(16π²), Σ a·exp(−b s²) then + c. */
double pdo_eval_gaussian(double q, const double *a, const double *b, size_t n, double c) {
    const double PI = 3.14159265358979323846;
    double s2 = q * q / (16.0 * PI * PI);
    double sum = 0.0;
    for (size_t i = 0; i < n; ++i) sum += a[i] * exp(-b[i] * s2);
    return sum + c;
}

/* src/formfactor.rs:378-385: Σ c_i q^i, q^i by repeated multiplication
 * (Rust's powi). */
double pdo_eval_polynomial(double q, const double *coeff, size_t n) {
    double sum = 0.0;
    for (size_t i = 0; i < n; ++i) {
        double p = 1.0;
        for (size_t e = 0; e < i; ++e) p *= q;
        sum += coeff[i] * p;
    }
    return sum;
}

/* src/formfactor.rs:388-408: binary search, exact hit returns the tabulated
 * value, otherwise linear interpolation in the bracketing interval. */
double pdo_interpolate(const double *xs, const double *ys, size_t n, double x) {
    size_t low = 0, high = n - 1;
    while (low < high) {
        size_t mid = (low + high) / 2;
        if (x < xs[mid]) high = mid;
        else if (x > xs[mid]) low = mid + 1;
        else return ys[mid];
    }
    double x0 = xs[low - 1], y0 = ys[low - 1], x1 = xs[low], y1 = ys[low];
    return y0 + (x - x0) * (y1 - y0) / (x1 - x0);
}

/* src/formfactor.rs:196 for the Fraser SingleGaussian built at
 * src/solvent/fraser.rs:48-57: F(q) = ρV·exp(−(V^{2/3}/denominator)·q·q). */
double pdo_fraser(double q, double volume, double rho, double denominator) {
    double a = rho * volume;
    double b = pow(volume, 2.0 / 3.0) / denominator;
    return a * exp(-b * q * q);
}

/* src/solvent/sasa.rs:54-59 for an atom whose whole shell is exposed:
 * 4π(r+probe)²·SHELL_THICKNESS/WATER_VOLUME (3 Å, 30 Å³). */
double pdo_sasa_full_weight(double radius, double probe) {
    const double PI = 3.14159265358979323846;
    double rp = radius + probe; /* powi(2) */
    double full = 4.0 * PI * (rp * rp);
    return full * 3.0 / 30.0;
}
