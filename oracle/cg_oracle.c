/*
 * cg_oracle.c -- CPU ORACLE for the cuGridder ms2dirty / dirty2ms path.
 *
 * THIS FILE IS TEST INFRASTRUCTURE.  It is a plain-C (C99 + OpenMP)
 * restatement of the reference algorithm (RapidsAtHKUST/cuGridder, improved
 * W-stacking) and of the FP64 direct DFT the reference's tests compare
 * against.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg may load it, and only as the checker; the product (libcugridder.so)
 * never links or calls it.
 *
 * Parity is pinned against outputs of the reference's own CUDA build
 * (compiled from its sources by oracle/ref.mk and run on a B200; the golden
 * outputs live in tests/golden/).
 *
 * Every function cites the reference file:line it restates.  Floating-point
 * operation order in the coordinate / bin-key path is kept exactly as in the
 * reference and this file is compiled with -ffp-contract=off, so the bin
 * keys are bit-identical to the reference's FP64 formulas.
 *
 * Complex arrays are interleaved (re, im) doubles.
 * Grid layout: fw[p][g1][g0], g0 fastest (size nf1), g1 (size nf2), p plane
 * (size nf3 = nw), exactly the reference's fw layout (conv.cu:596-598).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OG_PI 3.14159265358979323846
/* constants exactly as include/utils.h:29-30 */
#define OG_M_1_2PI 0.159154943091895336
#define OG_M_2PI 6.28318530717958648
#define OG_SPEEDOFLIGHT 299792458.0
#define OG_MAX_KW 16

typedef struct {
    int nrow, nx, ny;
    int N1, N2;              /* N1 = ny (grid dim 0), N2 = nx (grid dim 1): cugridder.cu:347 */
    double fov, freq, eps, sigma;
    int sign;
    int kw;                  /* kernel width W */
    double beta, es_c, es_halfwidth;
    int nf1, nf2, nf3;       /* grid sizes: nf1 <- N1, nf2 <- N2, nf3 = nw */
    double pixelsize_x, pixelsize_y;
    double i_center, i_half_width, o_center, o_half_width, gamma, h;
    int hivesize[3];         /* 8, 8, 1 (cuft.cu:253-264) */
    int nhive[3];
    /* gridding kernel: 0 = ES (the reference's), 1 = piecewise polynomial
     * (a learned kernel in Horner form, W segments x 8 coefficients) */
    int kern;
    double poly[OG_MAX_KW * 8];
} og_params;

/* kernel selected for the next og_setup (test infrastructure: not thread-safe) */
static int og_kern_kind = 0, og_kern_w = 0;
static double og_kern_poly[OG_MAX_KW * 8];

void og_set_kernel(int kind, int W, const double *coef)
{
    og_kern_kind = kind;
    og_kern_w = W;
    if (kind == 1) memcpy(og_kern_poly, coef, sizeof(double) * 8 * W);
}

/* piecewise polynomial: segment s = floor(d + W/2) at t = 2 (d + W/2 - s) - 1 */
static double og_poly_seg(const double *a, double t)
{
    double v = a[7];
    for (int n = 6; n >= 0; n--) v = v * t + a[n];
    return v;
}

static double og_poly_phi(const og_params *p, double d)
{
    double u = d + 0.5 * p->kw;
    int s = (int)floor(u);
    if (s < 0 || s >= p->kw) return 0.0;
    return og_poly_seg(p->poly + 8 * s, 2.0 * (u - s) - 1.0);
}

/* ---------------------------------------------------------------- */
/* next235beven: common_utils.cu:76-101                              */
int og_next235beven(int n, int b)
{
    if (n <= 2) return 2;
    if (n % 2 == 1) n += 1;
    int nplus = n - 2;
    int numdiv = 2;
    while ((numdiv > 1) || (nplus % b != 0)) {
        nplus += 2;
        numdiv = nplus;
        while (numdiv % 2 == 0) numdiv /= 2;
        while (numdiv % 3 == 0) numdiv /= 3;
        while (numdiv % 5 == 0) numdiv /= 5;
    }
    return nplus;
}

/* setup_conv_opts: conv_interp_invoker.cu:49-119 (FP64 build: EPSILON 1.1e-16,
 * utils.h:34-38; MAX_KERNEL_WIDTH 16, curafft_plan.h:14).  Returns ier. */
int og_setup_conv_opts(double eps, double upsampfac, int *kw_out, double *beta_out,
                       double *c_out, double *hw_out, double eps_floor)
{
    if (upsampfac != 2.0) {
        if (upsampfac <= 1.0) return 2;
    }
    int ier = 0;
    if (eps < eps_floor) { eps = eps_floor; ier = 1; }
    int kw = (int)ceil(-log10(eps / 10.0));
    if (upsampfac != 2.0)
        kw = (int)ceil(-log(eps) / (OG_PI * sqrt(1.0 - 1.0 / upsampfac)));
    if (kw < 2) kw = 2;
    if (kw > OG_MAX_KW) kw = OG_MAX_KW;
    double betaoverns = 2.30;
    if (kw == 2) betaoverns = 2.20;
    if (kw == 3) betaoverns = 2.26;
    if (kw == 4) betaoverns = 2.38;
    if (upsampfac != 2.0) {
        double gamma = 0.97;
        betaoverns = gamma * OG_PI * (1 - 1 / (2 * upsampfac));
    }
    *kw_out = kw;
    *hw_out = (double)kw / 2;
    *c_out = 4.0 / (double)(kw * kw);
    *beta_out = betaoverns * (double)kw;
    return ier;
}

/* get_num_cells: conv_interp_invoker.cu:30-47 */
int og_get_num_cells(int ms, double upsampfac, int kw)
{
    int nf = (int)(upsampfac * ms);
    if (nf < 2 * kw) nf = 2 * kw;
    if (nf < 1e11) nf = og_next235beven(nf, 1);
    return nf;
}

/* set_nhg_w: utils.cu:670-709 */
void og_set_nhg_w(double S, double X, int kw, double upsampfac, int *nf, double *h, double *gam)
{
    int nss = kw + 1;
    double Xsafe = X, Ssafe = S;
    if (X == 0.0) {
        if (S == 0.0) { Xsafe = 1.0; Ssafe = 1.0; }
        else Xsafe = (Xsafe > 1 / S) ? Xsafe : 1 / S;
    } else {
        Ssafe = (Ssafe > 1 / X) ? Ssafe : 1 / X;
    }
    double nfd = 2.0 * upsampfac * Ssafe * Xsafe / OG_PI + nss;
    if (!isfinite(nfd)) nfd = 0.0;
    int n = (int)nfd;
    n = n % 2 + n;
    if (n < 2 * kw) n = 2 * kw;
    *nf = n;
    *h = 2 * OG_PI / n;
    *gam = (double)n / (2.0 * upsampfac * Ssafe);
}

/* Effective coordinates, exact FP64 operation order of
 * get_effective_coordinate(...,sign) precomp.cu:48-72 followed by
 * rescaling_real (cugridder.cu:201-202) and the u/v swap of setup_plan
 * (cugridder.cu:191): grid dim 0 takes v*pixelsize_y, grid dim 1 takes
 * u*pixelsize_x, dim 2 takes w (scaled by sign). */
static inline void og_eff_coord(const double *uvw_row, double foc, int sign,
                                double pixx, double pixy,
                                double *x0, double *x1, double *w)
{
    double u = uvw_row[0], v = uvw_row[1], ww = uvw_row[2];
    u = u * foc;
    v = v * foc;
    ww = ww * (foc * (double)sign);
    u = u * (2 * OG_PI);
    v = v * (2 * OG_PI);
    ww = ww * (2 * OG_PI);
    u = u * pixx;
    v = v * pixy;
    *x0 = v;
    *x1 = u;
    *w = ww;
}

/* SHIFT_RESCALE(x, N, 0): conv.h:24 */
static inline double og_shift_rescale(double x, int N)
{
    double t = x - floor(x / OG_M_2PI) * OG_M_2PI;
    double s = t - (double)(t >= OG_PI) * OG_M_2PI;
    double X = (s * OG_M_1_2PI + 0.5) * N;
    /* a value rounding onto N (or below 0) is folded back into [0, N); the
     * reference keys such a row one hive row off -- a measure-zero case */
    if (X >= (double)N) X -= (double)N;
    if (X < 0.0) X += (double)N;
    return X;
}

/* Plan setup: gridder_setting + setup_gridder_plan (cugridder.cu:29-210).
 * w min/max as thrust get_max_min over the effective w (utils.cu:43-54). */
int og_setup(og_params *p, int nrow, int nx, int ny, double fov, double freq,
             const double *uvw, double eps, double sigma, int sign, double eps_floor)
{
    memset(p, 0, sizeof(*p));
    p->nrow = nrow; p->nx = nx; p->ny = ny;
    p->N1 = ny; p->N2 = nx;
    p->fov = fov; p->freq = freq; p->eps = eps; p->sigma = sigma; p->sign = sign;
    int ier = og_setup_conv_opts(eps, sigma, &p->kw, &p->beta, &p->es_c, &p->es_halfwidth, eps_floor);
    if (ier > 1) return ier;
    if (og_kern_kind == 1) {
        p->kern = 1;
        p->kw = og_kern_w;
        p->beta = 0; p->es_c = 0; p->es_halfwidth = og_kern_w / 2.0;
        memcpy(p->poly, og_kern_poly, sizeof(double) * 8 * og_kern_w);
    }
    p->pixelsize_x = fov / 180.0 * OG_PI / (double)p->N2;
    p->pixelsize_y = fov / 180.0 * OG_PI / (double)p->N1;
    double l_min = 0 - 0.5 * p->pixelsize_x * p->N2;
    double m_min = 0 - 0.5 * p->pixelsize_y * p->N1;
    double temp = 1.0 - pow(l_min, 2) - pow(m_min, 2);
    double n_lm = temp <= 0 ? 0 : sqrt(temp);
    double foc = freq / OG_SPEEDOFLIGHT;
    double wmax = -INFINITY, wmin = INFINITY;
    for (int i = 0; i < nrow; i++) {
        double a, b, w;
        og_eff_coord(uvw + 3 * (size_t)i, foc, sign, p->pixelsize_x, p->pixelsize_y, &a, &b, &w);
        if (w > wmax) wmax = w;
        if (w < wmin) wmin = w;
    }
    if (nrow == 0) { wmax = 0; wmin = 0; }
    p->i_center = (wmax + wmin) / 2.0;
    p->i_half_width = (wmax - wmin) / 2.0;
    double o_min = n_lm - 1;
    p->o_center = o_min / 2.0;
    p->o_half_width = fabs(o_min / 2.0);
    og_set_nhg_w(p->o_half_width, p->i_half_width, p->kw, sigma, &p->nf3, &p->h, &p->gamma);
    p->nf1 = og_get_num_cells(p->N1, sigma, p->kw);
    p->nf2 = og_get_num_cells(p->N2, sigma, p->kw);
    p->hivesize[0] = 8; p->hivesize[1] = 8; p->hivesize[2] = 1;
    p->nhive[0] = (p->nf1 - 1) / 8 + 1;
    p->nhive[1] = (p->nf2 - 1) / 8 + 1;
    p->nhive[2] = p->nf3;
    return ier;
}

/* Grid coordinates (in cells, [0,nf)) of every visibility, FP64:
 * effective coordinate -> pre_stage_2 (cuft.cu:82-104: w' = (w - i_c)/gamma)
 * -> SHIFT_RESCALE (conv.h:24). */
void og_grid_coords(const og_params *p, const double *uvw, double *X0, double *X1, double *X2)
{
    double foc = p->freq / OG_SPEEDOFLIGHT;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < p->nrow; i++) {
        double a, b, w;
        og_eff_coord(uvw + 3 * (size_t)i, foc, p->sign, p->pixelsize_x, p->pixelsize_y, &a, &b, &w);
        double wp = (w - p->i_center) / p->gamma;
        X0[i] = og_shift_rescale(a, p->nf1);
        X1[i] = og_shift_rescale(b, p->nf2);
        X2[i] = og_shift_rescale(wp, p->nf3);
    }
}

/* Hive-major cell key of histogram_3d_sparse (utils.cu:105-132) with the
 * 8x8x1 hive of method 6 (cuft.cu:253-258):
 * key = (hx + hy*nhx + hz*nhx*nhy)*64 + (bx%8) + (by%8)*8. */
static inline int64_t og_key(const og_params *p, double X0, double X1, double X2)
{
    int bx = (int)floor(X0), by = (int)floor(X1), bz = (int)floor(X2);
    int hx = bx / 8, hy = by / 8, hz = bz;
    int64_t h = (int64_t)hx + (int64_t)hy * p->nhive[0] + (int64_t)hz * p->nhive[0] * p->nhive[1];
    return h * 64 + (bx % 8) + (by % 8) * 8;
}

void og_bin_keys(const og_params *p, const double *uvw, int64_t *keys)
{
    double *X0 = malloc(sizeof(double) * (size_t)p->nrow * 3);
    double *X1 = X0 + p->nrow, *X2 = X1 + p->nrow;
    og_grid_coords(p, uvw, X0, X1, X2);
    for (int i = 0; i < p->nrow; i++) keys[i] = og_key(p, X0[i], X1[i], X2[i]);
    free(X0);
}

/* bin_mapping (conv_interp_invoker.cu:121-224): histogram per cell key,
 * exclusive scan (common_utils.cu:156-169), hive counts
 * (common_utils.cu:123-138) and the scatter of mapping_based_gather_3d
 * (utils.cu:457-486).  The reference's within-cell order is its atomicAdd
 * order; this restatement uses the stable (index) order, which is one of the
 * orders the reference can produce.
 *   hive_start: nhive0*nhive1*nhive2 + 1 ints (the reference's hive_count)
 *   perm:       nrow ints, perm[sorted position] = original index */
void og_bin_mapping(const og_params *p, const double *uvw, int64_t *hive_start, int *perm)
{
    int64_t nh = (int64_t)p->nhive[0] * p->nhive[1] * p->nhive[2];
    int64_t *keys = malloc(sizeof(int64_t) * (size_t)(p->nrow > 0 ? p->nrow : 1));
    og_bin_keys(p, uvw, keys);
    int64_t ncell = nh * 64;
    int64_t *cnt = calloc((size_t)ncell + 1, sizeof(int64_t));
    for (int i = 0; i < p->nrow; i++) cnt[keys[i]]++;
    int64_t run = 0;
    for (int64_t k = 0; k <= ncell; k++) { int64_t c = cnt[k]; cnt[k] = run; run += c; }
    for (int64_t hh = 0; hh <= nh; hh++) hive_start[hh] = cnt[hh * 64];
    for (int i = 0; i < p->nrow; i++) perm[cnt[keys[i]]++] = i;
    free(cnt);
    free(keys);
}

/* ---------------------------------------------------------------- */
/* Gauss-Legendre nodes/weights on [-1,1], own implementation (Newton
 * iteration on the three-term Legendre recurrence).  Nodes are returned in
 * decreasing order, so the first n/2 are the positive half; the reference's
 * fseries uses one half of the 2p nodes (deconv.cu:85-86), and since the
 * integrand is even either half gives the same sum. */
void og_gauss_legendre(int n, double *x, double *w)
{
    for (int k = 0; k < n; k++) {
        double z = cos(OG_PI * (k + 0.75) / (n + 0.5));
        double pp = 0;
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = z;
            for (int j = 2; j <= n; j++) {
                double p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p0) / j;
                p0 = p1; p1 = p2;
            }
            pp = n * (z * p1 - p0) / (z * z - 1.0);
            double dz = p1 / pp;
            z -= dz;
            if (fabs(dz) < 1e-16) break;
        }
        /* final derivative at the converged node */
        double p0 = 1.0, p1 = z;
        for (int j = 2; j <= n; j++) {
            double p2 = ((2.0 * j - 1.0) * z * p1 - (j - 1.0) * p0) / j;
            p0 = p1; p1 = p2;
        }
        pp = n * (z * p1 - p0) / (z * z - 1.0);
        x[k] = z;
        w[k] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
}

/* quadrature values g_n = alpha*w_n*phi(alpha*x_n), n < p, p = int(2+3*alpha):
 * deconv.cu:80-93 (func_type = kerevalmeth = 0, cugridder.cu:345). */
static int og_fseries_nodes(const og_params *p, double *xs, double *g)
{
    double alpha = p->kw / 2.0;
    int q = (int)(2 + 3.0 * alpha);
    double x[2 * 64], w[2 * 64];
    og_gauss_legendre(2 * q, x, w);
    for (int n = 0; n < q; n++) {
        double xn = x[n] * alpha;
        double phi = 0.0;
        if (p->kern)
            phi = og_poly_phi(p, xn);
        else if (fabs(xn) <= p->es_halfwidth)
            phi = exp(p->beta * (sqrt(1.0 - p->es_c * xn * xn) - 0));
        xs[n] = xn;
        g[n] = alpha * w[n] * phi;
    }
    return q;
}

/* fwkerhalf{1,2}: fourier_series_appro (deconv.cu:12-26) with N = nf/2+1;
 * the (-1)^k of the fftshift is folded into the cosine argument. */
void og_fseries_uv(const og_params *p, int nf, double *out)
{
    double xs[64], g[64];
    int q = og_fseries_nodes(p, xs, g);
    int N = nf / 2 + 1;
    for (int k = 0; k < N; k++) {
        double s = 0;
        for (int i = 0; i < q; i++) s += g[i] * cos((xs[i] - N + 1) / (double)(N - 1) * OG_PI * k);
        out[k] = 2 * s;
    }
}

/* z table of k_generation (precomp.cu:215-226) on the quarter image
 * (N2/2+1) x (N1/2+1), row <-> x pixel, col <-> y pixel. */
static inline double og_zq(const og_params *p, int row, int col)
{
    double t = 1.0 - pow(row * p->pixelsize_x, 2) - pow(col * p->pixelsize_y, 2);
    return t < 0 ? sqrt(-t) - 1 : sqrt(t) - 1;
}

/* fwkerhalf3 on the quarter image: pre_stage_2 (cuft.cu:82-104:
 * z' = (z - o_c)*gamma*h) then fourier_series_appro (deconv.cu:49-65). */
void og_fseries_w(const og_params *p, double *out_q, double *zp_q)
{
    double xs[64], g[64];
    int q = og_fseries_nodes(p, xs, g);
    int nr = p->N2 / 2 + 1, nc = p->N1 / 2 + 1;
    for (int r = 0; r < nr; r++)
        for (int c = 0; c < nc; c++) {
            double z = og_zq(p, r, c);
            double zp = (z - p->o_center) * p->gamma * p->h;
            double s = 0;
            for (int i = 0; i < q; i++) s += g[i] * 2 * cos(xs[i] * zp);
            out_q[r * nc + c] = s;
            if (zp_q) zp_q[r * nc + c] = zp;
        }
}

static inline double og_phi(const og_params *p, double d)
{
    if (fabs(d) >= p->kw / 2.0) return 0.0;
    return exp(p->beta * sqrt(1.0 - p->es_c * d * d));
}

/* taps of one coordinate: first tap index and the W kernel values
 * (|d| >= W/2 gives 0; conv.cu:591-618 uses strict |d| < W/2,
 * interp.cu:17-23 zeroes |d| >= W/2). */
static inline int og_taps(const og_params *p, double X, double *k)
{
    int x0 = (int)floor(X - p->kw / 2.0) + 1;
    if (p->kern) {
        /* tap i evaluates segment i at z = x0 + W/2 - X, z in (0, 1] */
        double t = 2.0 * ((double)x0 + p->kw / 2.0 - X) - 1.0;
        for (int i = 0; i < p->kw; i++) k[i] = og_poly_seg(p->poly + 8 * i, t);
        return x0;
    }
    for (int i = 0; i < p->kw; i++) k[i] = og_phi(p, (double)(x0 + i) - X);
    return x0;
}

static inline int og_wrap(int i, int n)
{
    i %= n;
    return i < 0 ? i + n : i;
}

/* Gridding (spreading), the periodic 3-D ES convolution computed by
 * conv_3d_outputdriven_t1 (conv.cu:522-627): fw[p][g1][g0] += c_j phi phi phi.
 * Parallel over bands of g1 rows (each thread owns its band). */
void og_grid(const og_params *p, const double *X0, const double *X1, const double *X2,
             const double *c, double *fw)
{
    size_t plane = (size_t)p->nf1 * p->nf2;
    memset(fw, 0, sizeof(double) * 2 * plane * p->nf3);
    int nth = 1;
#ifdef _OPENMP
    nth = omp_get_max_threads();
#endif
#pragma omp parallel num_threads(nth)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        int r0 = (int)((int64_t)p->nf2 * t / nth), r1 = (int)((int64_t)p->nf2 * (t + 1) / nth);
        double kx[OG_MAX_KW], ky[OG_MAX_KW], kz[OG_MAX_KW];
        for (int j = 0; j < p->nrow; j++) {
            int y0 = og_taps(p, X1[j], ky);
            int hit = 0;
            for (int b = 0; b < p->kw; b++) {
                int yy = og_wrap(y0 + b, p->nf2);
                if (yy >= r0 && yy < r1) { hit = 1; break; }
            }
            if (!hit) continue;
            int x0 = og_taps(p, X0[j], kx);
            int z0 = og_taps(p, X2[j], kz);
            double cr = c[2 * j], ci = c[2 * j + 1];
            for (int a = 0; a < p->kw; a++) {
                int zz = og_wrap(z0 + a, p->nf3);
                for (int b = 0; b < p->kw; b++) {
                    int yy = og_wrap(y0 + b, p->nf2);
                    if (yy < r0 || yy >= r1) continue;
                    double kzy = kz[a] * ky[b];
                    double *row = fw + 2 * ((size_t)zz * plane + (size_t)yy * p->nf1);
                    for (int e = 0; e < p->kw; e++) {
                        int xx = og_wrap(x0 + e, p->nf1);
                        double kv = kzy * kx[e];
                        row[2 * xx] += cr * kv;
                        row[2 * xx + 1] += ci * kv;
                    }
                }
            }
        }
    }
}

/* Degridding (interpolation), interp_3d_nputsdriven (interp.cu:132-210). */
void og_degrid(const og_params *p, const double *X0, const double *X1, const double *X2,
               const double *fw, double *c)
{
    size_t plane = (size_t)p->nf1 * p->nf2;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < p->nrow; j++) {
        double kx[OG_MAX_KW], ky[OG_MAX_KW], kz[OG_MAX_KW];
        int x0 = og_taps(p, X0[j], kx);
        int y0 = og_taps(p, X1[j], ky);
        int z0 = og_taps(p, X2[j], kz);
        double sr = 0, si = 0;
        for (int a = 0; a < p->kw; a++) {
            int zz = og_wrap(z0 + a, p->nf3);
            for (int b = 0; b < p->kw; b++) {
                int yy = og_wrap(y0 + b, p->nf2);
                double kzy = kz[a] * ky[b];
                const double *row = fw + 2 * ((size_t)zz * plane + (size_t)yy * p->nf1);
                for (int e = 0; e < p->kw; e++) {
                    int xx = og_wrap(x0 + e, p->nf1);
                    double kv = kzy * kx[e];
                    sr += row[2 * xx] * kv;
                    si += row[2 * xx + 1] * kv;
                }
            }
        }
        c[2 * j] = sr;
        c[2 * j + 1] = si;
    }
}

/* ---------------------------------------------------------------- */
/* Mixed-radix (2,3,4,5 and generic) recursive FFT, unnormalized:
 * out[k] = sum_n in[n*stride] exp(sign*2*pi*i*n*k/n_total) -- the cuFFT
 * convention of cufftExec*(..., CUFFT_INVERSE=+1 / CUFFT_FORWARD=-1)
 * used by cura_cufft (cuft.cu:192-212). */
typedef struct { int n; double *tw; } og_fft_plan;

static void og_fft_rec(const double *in, size_t stride, double *out, int n,
                       const double *tw, int twstep, int sign, double *scratch)
{
    if (n == 1) { out[0] = in[0]; out[1] = in[1]; return; }
    int r;
    if (n % 4 == 0) r = 4;
    else if (n % 2 == 0) r = 2;
    else if (n % 3 == 0) r = 3;
    else if (n % 5 == 0) r = 5;
    else r = n;
    int m = n / r;
    for (int q = 0; q < r; q++)
        og_fft_rec(in + 2 * q * stride, stride * r, out + 2 * q * m, m, tw, twstep * r, sign, scratch);
    /* butterflies: X[k + s*m] = sum_q W_n^{q(k+s m)} Y_q[k] */
    double *t = scratch;
    for (int k = 0; k < m; k++) {
        for (int q = 0; q < r; q++) {
            t[2 * q] = out[2 * (q * m + k)];
            t[2 * q + 1] = out[2 * (q * m + k) + 1];
        }
        for (int s = 0; s < r; s++) {
            double ar = 0, ai = 0;
            for (int q = 0; q < r; q++) {
                long e = ((long)q * (k + (long)s * m)) % n;
                double wr = tw[2 * e * twstep], wi = sign * tw[2 * e * twstep + 1];
                ar += t[2 * q] * wr - t[2 * q + 1] * wi;
                ai += t[2 * q] * wi + t[2 * q + 1] * wr;
            }
            out[2 * (k + s * m)] = ar;
            out[2 * (k + s * m) + 1] = ai;
        }
    }
}

/* in-place 1-D FFT of length n (contiguous), with twiddles for length n */
static void og_fft1d(double *data, int n, const double *tw, int sign, double *buf, double *scratch)
{
    memcpy(buf, data, sizeof(double) * 2 * n);
    og_fft_rec(buf, 1, data, n, tw, 1, sign, scratch);
}

static double *og_twiddles(int n)
{
    double *tw = malloc(sizeof(double) * 2 * n);
    for (int e = 0; e < n; e++) {
        tw[2 * e] = cos(2 * OG_PI * (double)e / n);
        tw[2 * e + 1] = sin(2 * OG_PI * (double)e / n);
    }
    return tw;
}

/* batched 2-D FFT of nf3 planes [nf2][nf1] (cuft.cu:20-44 plan, n={nf2,nf1}) */
void og_fft2_planes(const og_params *p, double *fw, int sign)
{
    int n1 = p->nf1, n2 = p->nf2;
    size_t plane = (size_t)n1 * n2;
    double *tw1 = og_twiddles(n1), *tw2 = og_twiddles(n2);
    int nmax = n1 > n2 ? n1 : n2;
    for (int pl = 0; pl < p->nf3; pl++) {
        double *P = fw + 2 * plane * pl;
#pragma omp parallel
        {
            double *buf = malloc(sizeof(double) * 2 * nmax);
            double *col = malloc(sizeof(double) * 2 * nmax);
            double *scr = malloc(sizeof(double) * 2 * nmax);
#pragma omp for schedule(static)
            for (int r = 0; r < n2; r++) og_fft1d(P + 2 * (size_t)r * n1, n1, tw1, sign, buf, scr);
#pragma omp for schedule(static)
            for (int cidx = 0; cidx < n1; cidx++) {
                for (int r = 0; r < n2; r++) {
                    col[2 * r] = P[2 * ((size_t)r * n1 + cidx)];
                    col[2 * r + 1] = P[2 * ((size_t)r * n1 + cidx) + 1];
                }
                og_fft1d(col, n2, tw2, sign, buf, scr);
                for (int r = 0; r < n2; r++) {
                    P[2 * ((size_t)r * n1 + cidx)] = col[2 * r];
                    P[2 * ((size_t)r * n1 + cidx) + 1] = col[2 * r + 1];
                }
            }
            free(buf); free(col); free(scr);
        }
    }
    free(tw1); free(tw2);
}

/* CMCL index map of deconv_2d (deconv.cu:268-272) */
static inline int og_cmcl(int k, int N, int nf)
{
    return k >= N / 2 ? k - N / 2 : nf + k - N / 2;
}

/* ---------------------------------------------------------------- */
/* Full ms2dirty (exec_vis2dirty, ra_exec.cu:184-468; flow 1):
 *   c *= wgt (ra_exec.cu:103-111), c *= e^{i o_c w} (pre_stage_1, cuft.cu:46-66),
 *   conv, FFT(+1), w_term_dft (cuft.cu:597-645), deconv_2d type 1
 *   (deconv.cu:250-294), w_term_deconv flag +1 (deconv.cu:401-432),
 *   div_n_lm (ra_exec.cu:23-37).
 * dirty: nx*ny complex, row-major [x][y].  Returns 0 or an error code. */
int og_ms2dirty(int nrow, int nx, int ny, double fov, double freq, const double *uvw,
                const double *vis, const double *wgt, double *dirty, double eps,
                double sigma, int sign, og_params *out_params)
{
    og_params P;
    int ier = og_setup(&P, nrow, nx, ny, fov, freq, uvw, eps, sigma, sign, 1.1e-16);
    if (ier > 1) return ier;
    if (out_params) *out_params = P;
    int N1 = P.N1, N2 = P.N2;
    size_t plane = (size_t)P.nf1 * P.nf2;
    double *X = malloc(sizeof(double) * 3 * (size_t)(nrow > 0 ? nrow : 1));
    double *c = malloc(sizeof(double) * 2 * (size_t)(nrow > 0 ? nrow : 1));
    og_grid_coords(&P, uvw, X, X + nrow, X + 2 * nrow);
    double foc = freq / OG_SPEEDOFLIGHT;
    for (int j = 0; j < nrow; j++) {
        double cr = vis[2 * j], ci = vis[2 * j + 1];
        if (wgt) { cr *= wgt[j]; ci *= wgt[j]; }
        if (P.o_center != 0) {
            double a, b, w;
            og_eff_coord(uvw + 3 * (size_t)j, foc, sign, P.pixelsize_x, P.pixelsize_y, &a, &b, &w);
            double ph = P.o_center * w * 1;
            double cs = cos(ph), sn = sin(ph);
            double tr = cr * cs - ci * sn, ti = cr * sn + ci * cs;
            cr = tr; ci = ti;
        }
        c[2 * j] = cr; c[2 * j + 1] = ci;
    }
    double *fw = malloc(sizeof(double) * 2 * plane * P.nf3);
    og_grid(&P, X, X + nrow, X + 2 * nrow, c, fw);
    og_fft2_planes(&P, fw, +1);
    double *k1 = malloc(sizeof(double) * (P.nf1 / 2 + 1));
    double *k2 = malloc(sizeof(double) * (P.nf2 / 2 + 1));
    og_fseries_uv(&P, P.nf1, k1);
    og_fseries_uv(&P, P.nf2, k2);
    int nc = N1 / 2 + 1;
    double *k3 = malloc(sizeof(double) * (size_t)nc * (N2 / 2 + 1));
    double *zp = malloc(sizeof(double) * (size_t)nc * (N2 / 2 + 1));
    og_fseries_w(&P, k3, zp);
    int nw = P.nf3;
#pragma omp parallel for schedule(static)
    for (int row = 0; row < N2; row++) {
        for (int col = 0; col < N1; col++) {
            int w1 = og_cmcl(col, N1, P.nf1), w2 = og_cmcl(row, N2, P.nf2);
            size_t idx_fw = (size_t)w1 + (size_t)w2 * P.nf1;
            int iq = abs(col - N1 / 2) + abs(row - N2 / 2) * nc;
            double z = zp[iq];
            double sr = 0, si = 0;
            for (int pl = 0; pl < nw; pl++) {
                double ph = z * (pl - nw / 2);
                double cs = cos(ph), sn = sin(ph);
                double fr = fw[2 * (idx_fw + plane * pl)], fi = fw[2 * (idx_fw + plane * pl) + 1];
                sr += fr * cs - fi * sn;
                si += fr * sn + fi * cs;
            }
            double kv = k1[abs(col - N1 / 2)] * k2[abs(row - N2 / 2)];
            sr /= kv; si /= kv;
            /* w_term_deconv, flag = +1 */
            double tmp = 1.0 - pow((row - N2 / 2) * P.pixelsize_x, 2) - pow((col - N1 / 2) * P.pixelsize_y, 2);
            double ph = (tmp < 0 ? (sqrt(-tmp) - 1) - P.o_center : (sqrt(tmp) - 1) - P.o_center) * P.i_center * 1;
            double cs = cos(ph), sn = sin(ph);
            double tr = (sr * cs - si * sn) / k3[iq], ti = (sr * sn + si * cs) / k3[iq];
            /* div_n_lm */
            double n_lm = sqrt(1.0 - pow((row - N2 / 2) * P.pixelsize_x, 2) - pow((col - N1 / 2) * P.pixelsize_y, 2));
            size_t o = (size_t)row * N1 + col;
            dirty[2 * o] = tr / n_lm;
            dirty[2 * o + 1] = ti / n_lm;
        }
    }
    free(X); free(c); free(fw); free(k1); free(k2); free(k3); free(zp);
    return 0;
}

/* Full dirty2ms (exec_dirty2vis, ra_exec.cu:470-680):
 *   fk /= n (div_n_lm), w_term_deconv flag -1, deconv_2d type 2 into plane 0,
 *   w_term_idft (cuft.cu:647-689), FFT(-1), interp, c *= wgt (the
 *   "divide" invoker multiplies, utils.cu:661-668), shift_corr flag -1
 *   (ra_exec.cu:55-66). */
int og_dirty2ms(int nrow, int nx, int ny, double fov, double freq, const double *uvw,
                double *vis, const double *wgt, const double *dirty, double eps,
                double sigma, int sign, og_params *out_params)
{
    og_params P;
    int ier = og_setup(&P, nrow, nx, ny, fov, freq, uvw, eps, sigma, sign, 1.1e-16);
    if (ier > 1) return ier;
    if (out_params) *out_params = P;
    int N1 = P.N1, N2 = P.N2;
    size_t plane = (size_t)P.nf1 * P.nf2;
    int nw = P.nf3;
    double *k1 = malloc(sizeof(double) * (P.nf1 / 2 + 1));
    double *k2 = malloc(sizeof(double) * (P.nf2 / 2 + 1));
    og_fseries_uv(&P, P.nf1, k1);
    og_fseries_uv(&P, P.nf2, k2);
    int nc = N1 / 2 + 1;
    double *k3 = malloc(sizeof(double) * (size_t)nc * (N2 / 2 + 1));
    double *zp = malloc(sizeof(double) * (size_t)nc * (N2 / 2 + 1));
    og_fseries_w(&P, k3, zp);
    double *fw = calloc(2 * plane * nw, sizeof(double));
#pragma omp parallel for schedule(static)
    for (int row = 0; row < N2; row++) {
        for (int col = 0; col < N1; col++) {
            size_t o = (size_t)row * N1 + col;
            double n_lm = sqrt(1.0 - pow((row - N2 / 2) * P.pixelsize_x, 2) - pow((col - N1 / 2) * P.pixelsize_y, 2));
            double fr = dirty[2 * o] / n_lm, fi = dirty[2 * o + 1] / n_lm;
            int iq = abs(col - N1 / 2) + abs(row - N2 / 2) * nc;
            double tmp = 1.0 - pow((row - N2 / 2) * P.pixelsize_x, 2) - pow((col - N1 / 2) * P.pixelsize_y, 2);
            double ph = (tmp < 0 ? (sqrt(-tmp) - 1) - P.o_center : (sqrt(tmp) - 1) - P.o_center) * P.i_center * (-1);
            double cs = cos(ph), sn = sin(ph);
            double tr = (fr * cs - fi * sn) / k3[iq], ti = (fr * sn + fi * cs) / k3[iq];
            double kv = k1[abs(col - N1 / 2)] * k2[abs(row - N2 / 2)];
            tr /= kv; ti /= kv;
            int w1 = og_cmcl(col, N1, P.nf1), w2 = og_cmcl(row, N2, P.nf2);
            size_t idx_fw = (size_t)w1 + (size_t)w2 * P.nf1;
            double z = zp[iq];
            for (int pl = 0; pl < nw; pl++) {
                double pph = -1 * z * (pl - nw / 2);
                double c2 = cos(pph), s2 = sin(pph);
                fw[2 * (idx_fw + plane * pl)] = tr * c2 - ti * s2;
                fw[2 * (idx_fw + plane * pl) + 1] = tr * s2 + ti * c2;
            }
        }
    }
    og_fft2_planes(&P, fw, -1);
    double *X = malloc(sizeof(double) * 3 * (size_t)(nrow > 0 ? nrow : 1));
    og_grid_coords(&P, uvw, X, X + nrow, X + 2 * nrow);
    og_degrid(&P, X, X + nrow, X + 2 * nrow, fw, vis);
    double foc = freq / OG_SPEEDOFLIGHT;
    for (int j = 0; j < nrow; j++) {
        double cr = vis[2 * j], ci = vis[2 * j + 1];
        if (wgt) { cr *= wgt[j]; ci *= wgt[j]; }
        double a, b, w;
        og_eff_coord(uvw + 3 * (size_t)j, foc, sign, P.pixelsize_x, P.pixelsize_y, &a, &b, &w);
        double wp = (w - P.i_center) / P.gamma;
        double ph = (wp * P.gamma + P.i_center) * P.o_center * (-1);
        double cs = cos(ph), sn = sin(ph);
        vis[2 * j] = cr * cs - ci * sn;
        vis[2 * j + 1] = cr * sn + ci * cs;
    }
    free(X); free(fw); free(k1); free(k2); free(k3); free(zp);
    return 0;
}

/* ---------------------------------------------------------------- */
/* FP64 direct DFT, the definition the reference's tests check against
 * (python/curagridder/test_wst.py:15-32, test/w_s_gridder_test.cu:257-291):
 *   dirty[x,y] = 1/n * sum_j wgt_j vis_j exp(i*2pi*f/c*(u l + v m + sign*w*(n-1)))
 * l = (x - nx/2)*fov/nx, m = (y - ny/2)*fov/ny (radians),
 * n - 1 = -(l^2+m^2)/(1+sqrt(1-l^2-m^2)).
 * npix < 0 computes every pixel; otherwise only pixel indices pix[0..npix). */
void og_dft_ms2dirty(int nrow, int nx, int ny, double fov, double freq, const double *uvw,
                     const double *vis, const double *wgt, int sign, int npix, const int64_t *pix,
                     double *out)
{
    double pixx = fov / 180.0 * OG_PI / nx, pixy = fov / 180.0 * OG_PI / ny;
    double s = 2 * OG_PI * freq / OG_SPEEDOFLIGHT;
    int64_t total = npix < 0 ? (int64_t)nx * ny : npix;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t q = 0; q < total; q++) {
        int64_t o = npix < 0 ? q : pix[q];
        int x = (int)(o / ny), y = (int)(o % ny);
        double l = (x - nx / 2) * pixx, m = (y - ny / 2) * pixy;
        double e2 = l * l + m * m;
        double nm1 = -e2 / (sqrt(1.0 - e2) + 1.0);
        double n = nm1 + 1;
        double sr = 0, si = 0;
        for (int j = 0; j < nrow; j++) {
            double ph = s * (uvw[3 * j] * l + uvw[3 * j + 1] * m + sign * uvw[3 * j + 2] * nm1);
            double cs = cos(ph), sn = sin(ph);
            double wr = vis[2 * j], wi = vis[2 * j + 1];
            if (wgt) { wr *= wgt[j]; wi *= wgt[j]; }
            sr += wr * cs - wi * sn;
            si += wr * sn + wi * cs;
        }
        out[2 * q] = sr / n;
        out[2 * q + 1] = si / n;
    }
}

/* adjoint DFT (test/w_s_degridder_test.cu:252-262 with the weight multiply
 * of cura_fw, ra_exec.cu:75-93):
 *   vis_j = wgt_j * sum_{x,y} dirty[x,y]/n exp(-i*2pi*f/c*(u l + v m + sign*w*(n-1)))
 * nvis < 0 computes every row; otherwise only rows rows[0..nvis). */
void og_dft_dirty2ms(int nrow, int nx, int ny, double fov, double freq, const double *uvw,
                     const double *dirty, const double *wgt, int sign, int nvis, const int64_t *rows,
                     double *out)
{
    double pixx = fov / 180.0 * OG_PI / nx, pixy = fov / 180.0 * OG_PI / ny;
    double s = 2 * OG_PI * freq / OG_SPEEDOFLIGHT;
    int64_t total = nvis < 0 ? nrow : nvis;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t q = 0; q < total; q++) {
        int64_t j = nvis < 0 ? q : rows[q];
        double sr = 0, si = 0;
        for (int x = 0; x < nx; x++) {
            double l = (x - nx / 2) * pixx;
            for (int y = 0; y < ny; y++) {
                double m = (y - ny / 2) * pixy;
                double e2 = l * l + m * m;
                double nm1 = -e2 / (sqrt(1.0 - e2) + 1.0);
                double n = nm1 + 1;
                double ph = -s * (uvw[3 * j] * l + uvw[3 * j + 1] * m + sign * uvw[3 * j + 2] * nm1);
                double cs = cos(ph), sn = sin(ph);
                size_t o = (size_t)x * ny + y;
                double dr = dirty[2 * o] / n, di = dirty[2 * o + 1] / n;
                sr += dr * cs - di * sn;
                si += dr * sn + di * cs;
            }
        }
        double w = wgt ? wgt[j] : 1.0;
        out[2 * q] = sr * w;
        out[2 * q + 1] = si * w;
    }
}

int og_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ---------------------------------------------------------------- */
/* Learned kernel family (no reference counterpart; checker of the CUDA
 * forward/backward kernels):
 *   phi(d) = exp(beta0 (sqrt(1 - t^2) - 1) + net(2 t^2 - 1)), t = 2d/W, |t| < 1,
 * net = w3 . tanh(W2 tanh(W1 x + b1) + b2) + b3, 32 hidden units per layer.
 * theta: W1[32], b1[32], W2[32][32] (row = output unit), b2[32], w3[32], b3. */
#define OG_H 32
static double og_net(const double *th, double x, double *h1, double *h2)
{
    const double *W1 = th, *b1 = th + OG_H, *W2 = th + 2 * OG_H, *b2 = W2 + OG_H * OG_H;
    const double *w3 = b2 + OG_H, *b3 = w3 + OG_H;
    for (int m = 0; m < OG_H; m++) h1[m] = tanh(W1[m] * x + b1[m]);
    double out = b3[0];
    for (int k = 0; k < OG_H; k++) {
        double a = b2[k];
        for (int m = 0; m < OG_H; m++) a += W2[k * OG_H + m] * h1[m];
        h2[k] = tanh(a);
        out += w3[k] * h2[k];
    }
    return out;
}

void og_learn_phi(const double *th, double beta0, int W, int n, const double *d, double *phi)
{
    for (int i = 0; i < n; i++) {
        double t = d[i] / (0.5 * W), t2 = t * t;
        if (!(t2 < 1.0)) { phi[i] = 0.0; continue; }
        double h1[OG_H], h2[OG_H];
        phi[i] = exp(beta0 * (sqrt(1.0 - t2) - 1.0) + og_net(th, 2.0 * t2 - 1.0, h1, h2));
    }
}

/* dtheta = sum_i dphi[i] * d phi(d[i]) / d theta (overwrites dtheta) */
void og_learn_phi_grad(const double *th, double beta0, int W, int n, const double *d,
                       const double *dphi, double *dtheta)
{
    const int NT = OG_H + OG_H + OG_H * OG_H + OG_H + OG_H + 1;
    const double *W2 = th + 2 * OG_H, *w3 = W2 + OG_H * OG_H + OG_H;
    double *gW1 = dtheta, *gb1 = dtheta + OG_H, *gW2 = dtheta + 2 * OG_H;
    double *gb2 = gW2 + OG_H * OG_H, *gw3 = gb2 + OG_H, *gb3 = gw3 + OG_H;
    memset(dtheta, 0, sizeof(double) * NT);
    for (int i = 0; i < n; i++) {
        double t = d[i] / (0.5 * W), t2 = t * t;
        if (!(t2 < 1.0)) continue;
        double x = 2.0 * t2 - 1.0, h1[OG_H], h2[OG_H], d2[OG_H];
        double out = og_net(th, x, h1, h2);
        double g = dphi[i] * exp(beta0 * (sqrt(1.0 - t2) - 1.0) + out);
        gb3[0] += g;
        for (int k = 0; k < OG_H; k++) {
            gw3[k] += g * h2[k];
            d2[k] = g * w3[k] * (1.0 - h2[k] * h2[k]);
            gb2[k] += d2[k];
            for (int m = 0; m < OG_H; m++) gW2[k * OG_H + m] += d2[k] * h1[m];
        }
        for (int m = 0; m < OG_H; m++) {
            double a = 0;
            for (int k = 0; k < OG_H; k++) a += d2[k] * W2[k * OG_H + m];
            a *= 1.0 - h1[m] * h1[m];
            gb1[m] += a;
            gW1[m] += a * x;
        }
    }
}
