// The exported C ABI of libcharm.so (declared in include/charm_b200.h).
//
// Argument checks, error reporting and output conventions restate CHarm
// 0.4.9 (files cited per function) so that callers see the same behaviour;
// the numerical work is delegated to the GPU engine (engine.cpp).
#include <cfloat>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include <cuda_runtime.h>

#include "../../include/charm_b200.h"
#include "engine.h"

extern "C"
{

// src/glob/glob.c:16-23
CHARM_EXTERN double charm_glob_threshold = 100.0 * DBL_EPSILON;
CHARM_EXTERN double charm_glob_threshold2 = 100000.0 * DBL_EPSILON;
CHARM_EXTERN unsigned long charm_glob_polar_optimization_a1 = 100;
CHARM_EXTERN double charm_glob_polar_optimization_a2 = -1.0;

// ---------------------------------------------------------------------------
// Error object, src/err/err_init.c, err_free.c, err_reset.c, err_isempty.c,
// err_handler.c, err_set.c
// ---------------------------------------------------------------------------
charm_err *charm_err_init(void)
{
    charm_err *err = (charm_err *)malloc(sizeof(charm_err));
    if (!err)
        return NULL;
    err->file = (char **)calloc(CHARM_ERR_MAX_LEVEL, sizeof(char *));
    err->line = (size_t *)calloc(CHARM_ERR_MAX_LEVEL, sizeof(size_t));
    err->func = (char **)calloc(CHARM_ERR_MAX_LEVEL, sizeof(char *));
    err->msg = (char *)calloc(CHARM_ERR_MAX_MSG, 1);
    bool ok = err->file && err->line && err->func && err->msg;
    for (size_t e = 0; ok && e < CHARM_ERR_MAX_LEVEL; e++)
    {
        err->file[e] = (char *)calloc(CHARM_ERR_MAX_FILE, 1);
        err->func[e] = (char *)calloc(CHARM_ERR_MAX_FUNC, 1);
        ok = err->file[e] && err->func[e];
    }
    if (!ok)
    {
        charm_err_free(err);
        return NULL;
    }
    err->distributed = 0;
    charm_err_reset(err);
    return err;
}

void charm_err_free(charm_err *err)
{
    if (!err)
        return;
    for (size_t e = 0; e < CHARM_ERR_MAX_LEVEL; e++)
    {
        if (err->file)
            free(err->file[e]);
        if (err->func)
            free(err->func[e]);
    }
    free(err->file);
    free(err->func);
    free(err->line);
    free(err->msg);
    free(err);
}

void charm_err_reset(charm_err *err)
{
    if (!err)
        return;
    err->level = 0;
    for (size_t e = 0; e < CHARM_ERR_MAX_LEVEL; e++)
    {
        memset(err->file[e], 0, CHARM_ERR_MAX_FILE);
        memset(err->func[e], 0, CHARM_ERR_MAX_FUNC);
    }
    memset(err->line, 0, CHARM_ERR_MAX_LEVEL * sizeof(size_t));
    err->code = CHARM_SUCCESS;
    memset(err->msg, 0, CHARM_ERR_MAX_MSG);
    err->saturated = 0;
}

_Bool charm_err_isempty(const charm_err *err)
{
    if (!err)
        return 0;
    return err->code == CHARM_SUCCESS;
}

// src/err/err_inc_level.c
static void err_inc_level(charm_err *err)
{
    if (err->saturated)
        return;
    err->level += 1;
    if (err->level >= CHARM_ERR_MAX_LEVEL)
        err->saturated = 1;
}

static void err_set(charm_err *err, const char *file, size_t line,
                    const char *func, int code, const char *msg)
{
    if (!err || err->saturated)
        return;
    size_t l = err->level;
    snprintf(err->file[l], CHARM_ERR_MAX_FILE, "%s", file);
    err->line[l] = line;
    snprintf(err->func[l], CHARM_ERR_MAX_FUNC, "%s", func);
    err->code = code;
    snprintf(err->msg, CHARM_ERR_MAX_MSG, "%s", msg);
    err_inc_level(err);
}

void charm_err_handler(charm_err *err, _Bool terminate)
{
    if (!err || charm_err_isempty(err))
        return;
    fprintf(stderr, "\n-----------\nCHarm ERROR\n-----------\n"
                    "Error code: %u                   Traceback (most recent "
                    "call last)\n\n",
            err->code);
    for (size_t e = err->level - 1; e != (size_t)(-1); e--)
        fprintf(stderr, "    File \"%s\", line: %zu, function: \"%s\"\n\n",
                err->file[e], err->line[e], err->func[e]);
    if (err->saturated)
        fprintf(stderr, "%s", "    Warning: The error structure is saturated.  "
                              "Most recent function calls may therefore not be "
                              "reported.\n\n");
    fprintf(stderr, "Error message: %s\n-----------\n", err->msg);
    if (terminate)
        exit(CHARM_FAILURE);
    charm_err_reset(err);
}

// src/misc/misc_is_nearly_equal.c:20-31
static bool nearly_equal(double a, double b, double eps)
{
    double aa = a < 0 ? -a : a, ba = b < 0 ? -b : b;
    double d = a > b ? a - b : b - a, s = aa + ba;
    if (a == b)
        return true;
    if (a == 0.0 || b == 0.0 || s == aa || s == ba)
        return d <= eps;
    return d / (aa > ba ? aa : ba) <= eps;
}

#define SET_ERR(err, code, msg) err_set((err), __FILE__, __LINE__, __func__, \
                                        (code), (msg))

// ---------------------------------------------------------------------------
// Points, src/crd/crd_point_alloc.c, crd_point_init.c, crd_point_free.c,
// crd_point_check_inputs.c, crd_point_npoint.c
// ---------------------------------------------------------------------------
static bool is_point_type(int t)
{
    return t == CHARM_CRD_POINT_SCATTERED || t == CHARM_CRD_POINT_GRID ||
           t == CHARM_CRD_POINT_GRID_GL || t == CHARM_CRD_POINT_GRID_DH1 ||
           t == CHARM_CRD_POINT_GRID_DH2;
}

static bool is_quad_type(int t)
{
    return t == CHARM_CRD_POINT_GRID_GL || t == CHARM_CRD_POINT_GRID_DH1 ||
           t == CHARM_CRD_POINT_GRID_DH2;
}

static bool is_grid_type(int t)
{
    return t == CHARM_CRD_POINT_GRID || is_quad_type(t);
}

charm_point *charm_crd_point_init(int type, size_t nlat, size_t nlon,
                                  double *lat, double *lon, double *r)
{
    if (!is_point_type(type))
        return NULL;
    if (type == CHARM_CRD_POINT_SCATTERED && nlat != nlon)
        return NULL;
    charm_point *p = (charm_point *)malloc(sizeof(charm_point));
    if (!p)
        return NULL;
    p->lat = p->lon = p->r = p->w = NULL;
    if (nlat > 0)
    {
        p->lat = lat;
        p->r = r;
    }
    if (nlon > 0)
        p->lon = lon;
    p->nlat = nlat;
    p->nlon = nlon;
    p->npoint = type == CHARM_CRD_POINT_SCATTERED ? nlat
                                                  : (is_grid_type(type)
                                                         ? nlat * nlon
                                                         : 0);
    p->type = type;
    p->owner = 0;
    p->distributed = 0;
    return p;
}

static charm_point *point_alloc(int type, size_t nlat, size_t nlon, bool zero)
{
    if (!is_point_type(type))
        return NULL;
    if (type == CHARM_CRD_POINT_SCATTERED && nlat != nlon)
        return NULL;
    double *lat = NULL, *lon = NULL, *r = NULL, *w = NULL;
    auto al = [&](size_t n) -> double * {
        return zero ? (double *)calloc(n, sizeof(double))
                    : (double *)malloc(n * sizeof(double));
    };
    charm_point *p = NULL;
    if (nlat > 0)
    {
        lat = al(nlat);
        r = al(nlat);
        if (!lat || !r)
            goto FAIL;
    }
    if (nlon > 0)
    {
        lon = al(nlon);
        if (!lon)
            goto FAIL;
    }
    p = charm_crd_point_init(type, nlat, nlon, lat, lon, r);
    if (!p)
        goto FAIL;
    if (is_quad_type(type))
    {
        w = al(nlat > 0 ? nlat : 1);
        if (!w)
            goto FAIL;
        p->w = w;
    }
    p->owner = 1;
    return p;
FAIL:
    free(lat);
    free(lon);
    free(r);
    free(w);
    free(p);
    return NULL;
}

charm_point *charm_crd_point_malloc(int type, size_t nlat, size_t nlon)
{
    return point_alloc(type, nlat, nlon, false);
}

charm_point *charm_crd_point_calloc(int type, size_t nlat, size_t nlon)
{
    return point_alloc(type, nlat, nlon, true);
}

void charm_crd_point_free(charm_point *pnt)
{
    if (!pnt)
        return;
    if (pnt->owner)
    {
        free(pnt->lat);
        free(pnt->lon);
        free(pnt->r);
        free(pnt->w);
    }
    free(pnt);
}

// src/crd/crd_point_gl_shape.c, crd_point_dh1_shape.c, crd_point_dh2_shape.c
void charm_crd_point_gl_shape(unsigned long nmax, size_t *nlat, size_t *nlon)
{
    *nlat = nmax + 1;
    *nlon = 2 * (nmax + 1);
}

void charm_crd_point_dh1_shape(unsigned long nmax, size_t *nlat, size_t *nlon)
{
    *nlat = 2 * (nmax + 1);
    *nlon = 2 * (nmax + 1);
}

void charm_crd_point_dh2_shape(unsigned long nmax, size_t *nlat, size_t *nlon)
{
    *nlat = 2 * (nmax + 1);
    *nlon = 4 * (nmax + 1);
}

// src/crd/crd_point_quad.c, crd_point_gl_chunk.c, crd_point_dh_chunk.c:
// NULL on any error (CHarm does not propagate the error object here).
static charm_point *quad_grid(int type, unsigned long nmax, double r)
{
    if (r <= 0.0)
        return NULL;
    size_t nlat, nlon;
    if (type == CHARM_CRD_POINT_GRID_GL)
        charm_crd_point_gl_shape(nmax, &nlat, &nlon);
    else if (type == CHARM_CRD_POINT_GRID_DH1)
        charm_crd_point_dh1_shape(nmax, &nlat, &nlon);
    else
        charm_crd_point_dh2_shape(nmax, &nlat, &nlon);
    charm_point *p = charm_crd_point_calloc(type, nlat, nlon);
    if (!p)
        return NULL;
    cb::Status st = cb::quad_nodes(type, nmax, p->lat, p->w);
    if (!st.ok())
    {
        charm_crd_point_free(p);
        return NULL;
    }
    for (size_t i = 0; i < nlat; i++)
        p->r[i] = r;
    const double PI = 3.14159265358979323846;
    double c = (type == CHARM_CRD_POINT_GRID_DH2) ? PI / (double)(2 * (nmax + 1))
                                                  : PI / (double)(nmax + 1);
    for (size_t j = 0; j < nlon; j++)
        p->lon[j] = c * (double)j;
    return p;
}

charm_point *charm_crd_point_gl(unsigned long nmax, double r)
{
    return quad_grid(CHARM_CRD_POINT_GRID_GL, nmax, r);
}

charm_point *charm_crd_point_dh1(unsigned long nmax, double r)
{
    return quad_grid(CHARM_CRD_POINT_GRID_DH1, nmax, r);
}

charm_point *charm_crd_point_dh2(unsigned long nmax, double r)
{
    return quad_grid(CHARM_CRD_POINT_GRID_DH2, nmax, r);
}

// ---------------------------------------------------------------------------
// Cells, src/crd/crd_cell_alloc.c, crd_cell_init.c, crd_cell_free.c,
// crd_cell_check_inputs.c
// ---------------------------------------------------------------------------
static bool is_cell_type(int t)
{
    return t == CHARM_CRD_CELL_GRID || t == CHARM_CRD_CELL_SCATTERED;
}

charm_cell *charm_crd_cell_init(int type, size_t nlat, size_t nlon,
                                double *latmin, double *latmax,
                                double *lonmin, double *lonmax, double *r)
{
    if (!is_cell_type(type))
        return NULL;
    if (type == CHARM_CRD_CELL_SCATTERED && nlat != nlon)
        return NULL;
    charm_cell *c = (charm_cell *)malloc(sizeof(charm_cell));
    if (!c)
        return NULL;
    c->latmin = c->latmax = c->lonmin = c->lonmax = c->r = NULL;
    if (nlat > 0)
    {
        c->latmin = latmin;
        c->latmax = latmax;
        c->r = r;
    }
    if (nlon > 0)
    {
        c->lonmin = lonmin;
        c->lonmax = lonmax;
    }
    c->nlat = nlat;
    c->nlon = nlon;
    c->ncell = type == CHARM_CRD_CELL_SCATTERED ? nlat : nlat * nlon;
    c->type = type;
    c->owner = 0;
    return c;
}

static charm_cell *cell_alloc(int type, size_t nlat, size_t nlon, bool zero)
{
    if (!is_cell_type(type))
        return NULL;
    if (type == CHARM_CRD_CELL_SCATTERED && nlat != nlon)
        return NULL;
    double *latmin = NULL, *latmax = NULL, *lonmin = NULL, *lonmax = NULL;
    double *r = NULL;
    auto al = [&](size_t n) -> double * {
        return zero ? (double *)calloc(n, sizeof(double))
                    : (double *)malloc(n * sizeof(double));
    };
    charm_cell *c = NULL;
    if (nlat > 0)
    {
        latmin = al(nlat);
        latmax = al(nlat);
        r = al(nlat);
        if (!latmin || !latmax || !r)
            goto FAIL;
    }
    if (nlon > 0)
    {
        lonmin = al(nlon);
        lonmax = al(nlon);
        if (!lonmin || !lonmax)
            goto FAIL;
    }
    c = charm_crd_cell_init(type, nlat, nlon, latmin, latmax, lonmin, lonmax,
                            r);
    if (!c)
        goto FAIL;
    c->owner = 1;
    return c;
FAIL:
    free(latmin);
    free(latmax);
    free(lonmin);
    free(lonmax);
    free(r);
    free(c);
    return NULL;
}

charm_cell *charm_crd_cell_malloc(int type, size_t nlat, size_t nlon)
{
    return cell_alloc(type, nlat, nlon, false);
}

charm_cell *charm_crd_cell_calloc(int type, size_t nlat, size_t nlon)
{
    return cell_alloc(type, nlat, nlon, true);
}

void charm_crd_cell_free(charm_cell *cell)
{
    if (!cell)
        return;
    if (cell->owner)
    {
        free(cell->latmin);
        free(cell->latmax);
        free(cell->lonmin);
        free(cell->lonmax);
        free(cell->r);
    }
    free(cell);
}

// ---------------------------------------------------------------------------
// Coefficients, src/shc/shc_alloc.c, shc_init.c, shc_init_chunk.c,
// shc_free.c
// ---------------------------------------------------------------------------
charm_shc *charm_shc_init(unsigned long nmax, double mu, double r, double *c,
                          double *s)
{
    if (r <= 0.0)
        return NULL;
    charm_shc *h = (charm_shc *)malloc(sizeof(charm_shc));
    if (!h)
        return NULL;
    h->nmax = nmax;
    h->mu = mu;
    h->r = r;
    size_t nmax1 = (size_t)nmax + 1;
    size_t len = ((nmax1 + 1) * nmax1) / 2;
    h->nc = h->ns = len;
    h->owner = 0;
    h->distributed = 0;
    h->c = (double **)malloc(nmax1 * sizeof(double *));
    h->s = (double **)malloc(nmax1 * sizeof(double *));
    if (!h->c || !h->s)
    {
        free(h->c);
        free(h->s);
        free(h);
        return NULL;
    }
    size_t idx = 0;
    for (size_t m = 0; m <= nmax; m++)
    {
        h->c[m] = c + idx;
        h->s[m] = s + idx;
        idx += nmax1 - m;
    }
    return h;
}

static charm_shc *shc_alloc(unsigned long nmax, double mu, double r, bool zero)
{
    size_t nmax1 = (size_t)nmax + 1;
    size_t len = ((nmax1 + 1) * nmax1) / 2;
    double *c = zero ? (double *)calloc(len, sizeof(double))
                     : (double *)malloc(len * sizeof(double));
    double *s = zero ? (double *)calloc(len, sizeof(double))
                     : (double *)malloc(len * sizeof(double));
    charm_shc *h = NULL;
    if (!c || !s)
        goto FAIL;
    h = charm_shc_init(nmax, mu, r, c, s);
    if (!h)
        goto FAIL;
    h->owner = 1;
    return h;
FAIL:
    free(c);
    free(s);
    return NULL;
}

charm_shc *charm_shc_malloc(unsigned long nmax, double mu, double r)
{
    return shc_alloc(nmax, mu, r, false);
}

charm_shc *charm_shc_calloc(unsigned long nmax, double mu, double r)
{
    return shc_alloc(nmax, mu, r, true);
}

void charm_shc_free(charm_shc *shcs)
{
    if (!shcs)
        return;
    if (shcs->owner && shcs->c && shcs->s)
    {
        free(shcs->c[0]);
        free(shcs->s[0]);
    }
    free(shcs->c);
    free(shcs->s);
    free(shcs);
}

// ---------------------------------------------------------------------------
// Synthesis, src/shs/shs_point.c:26-129, shs_point_gradn.c:32-165,
// shs_point_guru.c:21-119
// ---------------------------------------------------------------------------
static void report(charm_err *err, const char *func, const cb::Status &st)
{
    if (!st.ok())
        err_set(err, __FILE__, __LINE__, func, st.code, st.msg.c_str());
}

static bool check_nmax(const charm_shc *shcs, unsigned long nmax,
                       charm_err *err, const char *what)
{
    if (nmax > shcs->nmax)
    {
        char msg[CHARM_ERR_MAX_MSG];
        snprintf(msg, sizeof msg,
                 "Maximum harmonic degree of the %s \"nmax = %lu\" cannot be "
                 "larger than maximum harmonic degree of spherical harmonic "
                 "coefficients \"shcs->nmax = %lu\".",
                 what, nmax, shcs->nmax);
        SET_ERR(err, CHARM_EFUNCARG, msg);
        return false;
    }
    return true;
}

static bool check_type_shs(const charm_point *pnt, charm_err *err)
{
    if (pnt->type != CHARM_CRD_POINT_SCATTERED && !is_grid_type(pnt->type))
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "Unsupported \"pnt->type\" for spherical harmonic synthesis "
                "of point values.");
        return false;
    }
    if (pnt->type == CHARM_CRD_POINT_SCATTERED && pnt->nlat != pnt->nlon)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "The number of latitudes and longitudes in the \"pnt\" "
                "structure must be the same to perform point-wise spherical "
                "harmonic synthesis.");
        return false;
    }
    return true;
}

void charm_shs_point(const charm_point *pnt, const charm_shc *shcs,
                     unsigned long nmax, double *f, charm_err *err)
{
    if (!check_nmax(shcs, nmax, err, "synthesis"))
        return;
    if (!check_type_shs(pnt, err))
        return;
    if (pnt->npoint == 0)
        return;
    double *fp[1] = {f};
    report(err, __func__, cb::shs_point(pnt, shcs, nmax, 0, 0, 0, 0, fp));
}

void charm_shs_point_grad1(const charm_point *pnt, const charm_shc *shcs,
                           unsigned long nmax, double **f, charm_err *err)
{
    if (!check_nmax(shcs, nmax, err, "synthesis"))
        return;
    if (!check_type_shs(pnt, err))
        return;
    if (pnt->npoint == 0)
        return;
    cb::Status st = cb::shs_point(pnt, shcs, nmax, 1, 1, 1, 1, f);
    report(err, __func__, st);
    if (!st.ok())
        return;
    // src/shs/shs_point_gradn.c:133-145: f holds l, r, p; reorder to x, y, z
    double *fx = f[2], *fy = f[0], *fz = f[1];
    f[0] = fx;
    f[1] = fy;
    f[2] = fz;
}

void charm_shs_point_grad2(const charm_point *pnt, const charm_shc *shcs,
                           unsigned long nmax, double **f, charm_err *err)
{
    if (!check_nmax(shcs, nmax, err, "synthesis"))
        return;
    if (!check_type_shs(pnt, err))
        return;
    if (pnt->npoint == 0)
        return;
    cb::Status st = cb::shs_point(pnt, shcs, nmax, 2, 2, 2, 2, f);
    report(err, __func__, st);
    if (!st.ok())
        return;
    // src/shs/shs_point_gradn.c:146-165: ll lr lp rr rp pp -> xx xy xz yy yz zz
    double *fxx = f[5], *fxy = f[2], *fxz = f[4];
    double *fyy = f[0], *fyz = f[1], *fzz = f[3];
    f[0] = fxx;
    f[1] = fxy;
    f[2] = fxz;
    f[3] = fyy;
    f[4] = fyz;
    f[5] = fzz;
}

void charm_shs_point_guru(const charm_point *pnt, const charm_shc *shcs,
                          unsigned long nmax, unsigned dr, unsigned dlat,
                          unsigned dlon, double *f, charm_err *err)
{
    if (!check_nmax(shcs, nmax, err, "synthesis"))
        return;
    // src/shs/shs_check_single_derivative.c
    if ((int)dr < 0 || (int)dlat < 0 || (int)dlon < 0 || dr + dlat + dlon > 2)
    {
        char msg[CHARM_ERR_MAX_MSG];
        snprintf(msg, sizeof msg,
                 "The sum \"dr + dlat + dlon\" is \"%d\", but it cannot be "
                 "larger than \"%d\".",
                 (int)(dr + dlat + dlon), 2);
        SET_ERR(err, CHARM_EFUNCARG, msg);
        return;
    }
    if (pnt->npoint == 0)
        return;
    if (!check_type_shs(pnt, err))
        return;
    double *fp[1] = {f};
    report(err, __func__,
           cb::shs_point(pnt, shcs, nmax, 0, (int)dr, (int)dlat, (int)dlon, fp));
}

// ---------------------------------------------------------------------------
// Analysis, src/sha/sha_point.c:124-206
// ---------------------------------------------------------------------------
void charm_sha_point(const charm_point *pnt, const double *f,
                     unsigned long nmax, charm_shc *shcs, charm_err *err)
{
    if (!check_nmax(shcs, nmax, err, "analysis"))
        return;
    if (!is_quad_type(pnt->type))
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "Unsupported \"pnt->type\" for spherical harmonic analysis of "
                "point data values.");
        return;
    }
    const double r0 = pnt->r[0];
    for (size_t i = 1; i < pnt->nlat; i++)
    {
        if (!nearly_equal(pnt->r[i], r0, charm_glob_threshold))
        {
            SET_ERR(err, CHARM_EFUNCARG,
                    "All spherical radii in \"pnt->r\" must be equal.");
            return;
        }
    }
    unsigned long nmax_grd = pnt->type == CHARM_CRD_POINT_GRID_GL
                                 ? (unsigned long)pnt->nlat - 1
                                 : ((unsigned long)pnt->nlat - 2) / 2;
    if (nmax > nmax_grd)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "The input data grid \"pnt\" was created for a maximum degree "
                "that is not high enough to recover harmonics up to the "
                "specified maximum degree of the analysis.");
        return;
    }
    report(err, __func__, cb::sha_point(pnt, f, nmax, shcs));
}

// ---------------------------------------------------------------------------
// Coefficient files in CHarm's binary format: src/shc/shc_read_bin.c:18-256,
// src/shc/shc_write_bin.c:18-187 (same checks, messages and return values)
// ---------------------------------------------------------------------------
unsigned long charm_shc_read_bin(const char *pathname, unsigned long nmax,
                                 charm_shc *shcs, charm_err *err)
{
    const bool nmax_only = nmax == CHARM_SHC_NMAX_MODEL && shcs == NULL;
    FILE *fp = fopen(pathname, "rb");
    if (!fp)
    {
        char msg[CHARM_ERR_MAX_MSG];
        snprintf(msg, sizeof msg, "Couldn't open \"%s\".", pathname);
        SET_ERR(err, CHARM_EFILEIO, msg);
        return CHARM_SHC_NMAX_ERROR;
    }
    unsigned long nmax_file = CHARM_SHC_NMAX_ERROR;
    double mu = 0.0, r = 0.0;
    if (fread(&nmax_file, sizeof nmax_file, 1, fp) != 1)
    {
        SET_ERR(err, CHARM_EFILEIO,
                "Failed to read the maximum harmonic degree.");
        goto EXIT;
    }
    if (nmax_only)
        goto EXIT;
    if (fread(&mu, sizeof mu, 1, fp) != 1)
    {
        SET_ERR(err, CHARM_EFILEIO, "Failed to read the scaling parameter.");
        goto EXIT;
    }
    if (fread(&r, sizeof r, 1, fp) != 1)
    {
        SET_ERR(err, CHARM_EFILEIO,
                "Failed to read the radius of the reference sphere.");
        goto EXIT;
    }
    if (nmax > nmax_file)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "Not enough coefficients in the input file for the maximum "
                "harmonic degree \"nmax\".");
        goto EXIT;
    }
    if (shcs->nmax < nmax)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "Too low maximum degree \"shcs->nmax\" to read coefficients "
                "up to degree \"nmax\".");
        goto EXIT;
    }
    shcs->mu = mu;
    shcs->r = r;
    memset(shcs->c[0], 0, shcs->nc * sizeof(double));
    memset(shcs->s[0], 0, shcs->ns * sizeof(double));
    for (int part = 0; part < 2; part++)
    {
        // column m of the file holds nmax_file + 1 - m values; the first
        // nmax + 1 - m of the columns m <= nmax are kept
        bool ok = true;
        for (unsigned long m = 0; ok && m <= nmax_file; m++)
        {
            const long len = (long)(nmax_file + 1 - m);
            if (m <= nmax)
            {
                double *col = part ? shcs->s[m] : shcs->c[m];
                const size_t nread = (size_t)(nmax + 1 - m);
                ok = fread(col, sizeof(double), nread, fp) == nread &&
                     fseek(fp, (len - (long)nread) * (long)sizeof(double),
                           SEEK_CUR) == 0;
            }
            else
                ok = fseek(fp, len * (long)sizeof(double), SEEK_CUR) == 0;
        }
        if (!ok)
        {
            SET_ERR(err, CHARM_EFILEIO,
                    part ? "Failed to read the \"S\" coefficients."
                         : "Failed to read the \"C\" coefficients.");
            goto EXIT;
        }
    }
EXIT:
    fclose(fp);
    return nmax_file;
}

void charm_shc_write_bin(const charm_shc *shcs, unsigned long nmax,
                         const char *pathname, charm_err *err)
{
    FILE *fp = fopen(pathname, "wb");
    if (!fp)
    {
        char msg[CHARM_ERR_MAX_MSG];
        snprintf(msg, sizeof msg, "Couldn't create \"%s\".", pathname);
        SET_ERR(err, CHARM_EFILEIO, msg);
        return;
    }
    if (nmax > shcs->nmax)
        SET_ERR(err, CHARM_EFUNCARG,
                "Not enough coefficients in \"shcs\" to write up to degree "
                "\"nmax\".");
    else if (fwrite(&nmax, sizeof nmax, 1, fp) != 1)
        SET_ERR(err, CHARM_EFILEIO,
                "Failed to write the maximum harmonic degree.");
    else if (fwrite(&shcs->mu, sizeof(double), 1, fp) != 1)
        SET_ERR(err, CHARM_EFILEIO, "Failed to write the scaling parameter.");
    else if (fwrite(&shcs->r, sizeof(double), 1, fp) != 1)
        SET_ERR(err, CHARM_EFILEIO,
                "Failed to write the radius of the reference sphere.");
    else
    {
        for (int part = 0; part < 2; part++)
        {
            bool ok = true;
            for (unsigned long m = 0; ok && m <= nmax; m++)
            {
                const double *col = part ? shcs->s[m] : shcs->c[m];
                const size_t n = (size_t)(nmax + 1 - m);
                ok = fwrite(col, sizeof(double), n, fp) == n;
            }
            if (!ok)
            {
                SET_ERR(err, CHARM_EFILEIO,
                        part ? "Failed to write the \"S\" coefficients)."
                             : "Failed to write the \"C\" coefficients).");
                break;
            }
        }
    }
    fclose(fp);
}

// ---------------------------------------------------------------------------
// Global spectral gravity forward modelling: src/gfm/gfm_sgfm.c (checks in
// CHarm's order and wording), gfm_global_density_lateral.c,
// gfm_global_density_3d.c, gfm_global_density_const.c
// ---------------------------------------------------------------------------
static void gfm_run(const charm_shc *shape_shcs, unsigned long shape_nmax,
                    double R, charm_shc **density_shcs,
                    unsigned long *density_nmax, unsigned density_order,
                    double rho, double G, double mass, unsigned pmin,
                    unsigned pmax, unsigned long nmax_pot,
                    const char *hro_path, const char *pot_path,
                    const char *fmt, charm_shc *pot, charm_err *err,
                    const char *func)
{
    char msg[CHARM_ERR_MAX_MSG];
    const double thr = charm_glob_threshold;
    if (shape_nmax > shape_shcs->nmax)
    {
        snprintf(msg, sizeof msg,
                 "\"shape_nmax\" is \"%lu\", but it cannot be larger than "
                 "\"shape_shcs->nmax = %lu\".",
                 shape_nmax, shape_shcs->nmax);
        SET_ERR(err, CHARM_EFUNCARG, msg);
        return;
    }
    if (!nearly_equal(shape_shcs->mu, 1.0, thr))
    {
        snprintf(msg, sizeof msg,
                 "\"shape_shcs->mu\" is \"%0.16e\", but it has to be \"1.0\".",
                 shape_shcs->mu);
        SET_ERR(err, CHARM_EFUNCARG, msg);
        return;
    }
    if (!nearly_equal(shape_shcs->r, 1.0, thr))
    {
        snprintf(msg, sizeof msg,
                 "\"shape_shcs->r\" is \"%0.16e\", but it has to be \"1.0\".",
                 shape_shcs->r);
        SET_ERR(err, CHARM_EFUNCARG, msg);
        return;
    }
    if (R <= 0.0)
    {
        snprintf(msg, sizeof msg,
                 "\"shape_ref_radius\" is \"%0.16e\", but it has to be "
                 "positive.", R);
        SET_ERR(err, CHARM_EFUNCARG, msg);
        return;
    }
    if (nearly_equal(mass, 0.0, thr))
    {
        SET_ERR(err, CHARM_EFUNCARG, "\"mass\" cannot be zero.");
        return;
    }
    // src/gfm/gfm_check_p.c
    if (pmin < 1 || pmax < 1)
    {
        SET_ERR(err, CHARM_EFUNCARG, "Topography power must be positive.");
        return;
    }
    if (pmin > pmax)
    {
        snprintf(msg, sizeof msg,
                 "\"shape_power_min\" is \"%u\", but it cannot be larger than "
                 "\"shape_power_max = %u\".", pmin, pmax);
        SET_ERR(err, CHARM_EFUNCARG, msg);
        return;
    }
    for (unsigned i = 0; density_shcs && i <= density_order; i++)
    {
        if (density_nmax[i] > density_shcs[i]->nmax)
        {
            snprintf(msg, sizeof msg,
                     "\"density_nmax[%u]\" is \"%lu\", but it cannot be larger "
                     "than \"density_shcs[%u]->nmax = %lu\".",
                     i, density_nmax[i], i, density_shcs[i]->nmax);
            SET_ERR(err, CHARM_EFUNCARG, msg);
            return;
        }
        if (!nearly_equal(density_shcs[i]->mu, 1.0, thr))
        {
            snprintf(msg, sizeof msg,
                     "\"density_shcs[%u]->mu\" is \"%0.16e\", but it has to "
                     "be \"1.0\".", i, density_shcs[i]->mu);
            SET_ERR(err, CHARM_EFUNCARG, msg);
            return;
        }
        if (!nearly_equal(density_shcs[i]->r, 1.0, thr))
        {
            snprintf(msg, sizeof msg,
                     "\"density_shcs[%u]->r\" is \"%0.16e\", but it has to "
                     "be \"1.0\".", i, density_shcs[i]->r);
            SET_ERR(err, CHARM_EFUNCARG, msg);
            return;
        }
    }
    if (pot && nmax_pot > pot->nmax)
    {
        snprintf(msg, sizeof msg,
                 "\"potential_shcs_nmax\" is \"%lu\", but it cannot be larger "
                 "than \"potential_shcs->nmax = %lu\".", nmax_pot, pot->nmax);
        SET_ERR(err, CHARM_EFUNCARG, msg);
        return;
    }
    if (hro_path || pot_path)
    {
        if (!fmt || (strcmp(fmt, "bin") && strcmp(fmt, "mtx") &&
                     strcmp(fmt, "tbl") && strcmp(fmt, "dov")))
        {
            SET_ERR(err, CHARM_EFUNCARG,
                    "Unsupported value of \"shcs_file_format\".");
            return;
        }
        if (strcmp(fmt, "bin"))
        {
            SET_ERR(err, CHARM_EFUNCARG,
                    "This library exports the partial coefficients in the "
                    "\"bin\" format only.");
            return;
        }
    }
    cb::GfmArgs g{};
    g.shape = shape_shcs;
    g.shape_nmax = shape_nmax;
    g.R = R;
    g.density = density_shcs;
    g.density_nmax = density_nmax;
    g.density_order = density_order;
    g.rho = rho;
    g.G = G;
    g.mass = mass;
    g.pmin = pmin;
    g.pmax = pmax;
    g.nmax_pot = nmax_pot;
    g.hro_path = hro_path;
    g.pot_path = pot_path;
    g.pot = pot;
    report(err, func, cb::gfm_global(g));
}

void charm_gfm_global_density_3d(const charm_shc *shape_shcs,
                                 unsigned long shape_nmax,
                                 double shape_radius_ref,
                                 charm_shc **density_shcs,
                                 unsigned long *density_nmax,
                                 unsigned density_order, double grav_const,
                                 double mass, unsigned shape_power_min,
                                 unsigned shape_power_max,
                                 unsigned long potential_shcs_nmax,
                                 const char *shape_density_shcs_path,
                                 const char *potential_shcs_path,
                                 const char *shcs_file_format,
                                 charm_shc *potential_shcs, charm_err *err)
{
    gfm_run(shape_shcs, shape_nmax, shape_radius_ref, density_shcs,
            density_nmax, density_order, 0.0, grav_const, mass,
            shape_power_min, shape_power_max, potential_shcs_nmax,
            shape_density_shcs_path, potential_shcs_path, shcs_file_format,
            potential_shcs, err, __func__);
}

void charm_gfm_global_density_lateral(
    const charm_shc *shape_shcs, unsigned long shape_nmax,
    double shape_radius_ref, charm_shc *density_shcs,
    unsigned long density_nmax, double grav_const, double mass,
    unsigned shape_power_min, unsigned shape_power_max,
    unsigned long potential_shcs_nmax, const char *shape_density_shcs_path,
    const char *potential_shcs_path, const char *shcs_file_format,
    charm_shc *potential_shcs, charm_err *err)
{
    // src/gfm/gfm_global_density_lateral.c:30-60
    if (density_nmax > density_shcs->nmax)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "\"density_nmax\" cannot be larger than "
                "\"density_shcs->nmax\".");
        return;
    }
    if (!nearly_equal(density_shcs->mu, 1.0, charm_glob_threshold))
    {
        SET_ERR(err, CHARM_EFUNCARG, "\"density_shcs->mu\" have to be \"1.0\".");
        return;
    }
    if (!nearly_equal(density_shcs->r, 1.0, charm_glob_threshold))
    {
        SET_ERR(err, CHARM_EFUNCARG, "\"density_shcs->r\" have to be \"1.0\".");
        return;
    }
    gfm_run(shape_shcs, shape_nmax, shape_radius_ref, &density_shcs,
            &density_nmax, 0, 0.0, grav_const, mass, shape_power_min,
            shape_power_max, potential_shcs_nmax, shape_density_shcs_path,
            potential_shcs_path, shcs_file_format, potential_shcs, err,
            __func__);
}

void charm_gfm_global_density_const(
    const charm_shc *shape_shcs, unsigned long shape_nmax,
    double shape_radius_ref, double density, double grav_const, double mass,
    unsigned shape_power_min, unsigned shape_power_max,
    unsigned long potential_shcs_nmax, const char *shape_shcs_path,
    const char *potential_shcs_path, const char *shcs_file_format,
    charm_shc *potential_shcs, charm_err *err)
{
    gfm_run(shape_shcs, shape_nmax, shape_radius_ref, nullptr, nullptr, 0,
            density, grav_const, mass, shape_power_min, shape_power_max,
            potential_shcs_nmax, shape_shcs_path, potential_shcs_path,
            shcs_file_format, potential_shcs, err, __func__);
}

// ---------------------------------------------------------------------------
// Cells: src/shs/shs_cell.c:22-121, src/sha/sha_cell.c:37-100
// ---------------------------------------------------------------------------
static bool check_nmax_cell(const charm_shc *shcs, unsigned long nmax,
                            charm_err *err, const char *what)
{
    if (nmax > shcs->nmax)
    {
        char msg[CHARM_ERR_MAX_MSG];
        snprintf(msg, sizeof msg,
                 "Maximum harmonic degree of the %s (\"nmax\") cannot be "
                 "larger than maximum harmonic degree of spherical harmonic "
                 "coefficients (\"shcs->nmax\").",
                 what);
        SET_ERR(err, CHARM_EFUNCARG, msg);
        return false;
    }
    return true;
}

static bool check_type_shs_cell(const charm_cell *cell, charm_err *err)
{
    if (cell->type == CHARM_CRD_CELL_SCATTERED)
    {
        if (cell->nlat != cell->nlon)
        {
            SET_ERR(err, CHARM_EFUNCARG,
                    "The number of latitudes and longitudes in the \"cell\" "
                    "structure must be the same in order to perform "
                    "cell-wise spherical harmonic synthesis.");
            return false;
        }
        return true;
    }
    if (cell->type != CHARM_CRD_CELL_GRID)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "Unsupported \"cell->type\" for spherical harmonic synthesis "
                "of block-mean values in cells.");
        return false;
    }
    return true;
}

void charm_shs_cell(const charm_cell *cell, const charm_shc *shcs,
                    unsigned long nmax, double *f, charm_err *err)
{
    if (!check_nmax_cell(shcs, nmax, err, "synthesis"))
        return;
    if (cell->ncell == 0)
        return;
    if (!check_type_shs_cell(cell, err))
        return;
    report(err, __func__, cb::shs_cell(cell, shcs, nmax, f));
}

static bool check_sha_cell(const charm_cell *cell, int method,
                           charm_err *err)
{
    if (method != CHARM_SHA_CELL_AQ)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "Unsupported \"method\" of spherical harmonic analysis of "
                "block-mean data values.");
        return false;
    }
    if (cell->type != CHARM_CRD_CELL_GRID)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "Unsupported \"cell->type\" for spherical harmonic analysis "
                "of block-mean data values.");
        return false;
    }
    return true;
}

void charm_sha_cell(const charm_cell *cell, const double *f,
                    unsigned long nmax, int method, charm_shc *shcs,
                    charm_err *err)
{
    if (!check_sha_cell(cell, method, err))
        return;
    if (!check_nmax_cell(shcs, nmax, err, "analysis"))
        return;
    if (cell->ncell == 0)
        return;
    report(err, __func__, cb::sha_cell(cell, f, nmax, shcs));
}

} // extern "C"

// ---------------------------------------------------------------------------
// Extensions (include/charm_b200.h): device-resident calls and measurement
// hooks.  They have no counterpart in CHarm's API.
// ---------------------------------------------------------------------------
extern "C"
{

void charm_b200_shs_point_dev(const charm_point *pnt, unsigned long shc_nmax,
                              double mu, double r, const double *d_c,
                              const double *d_s, unsigned long nmax,
                              int kgrad, unsigned dr, unsigned dlat,
                              unsigned dlon, double *d_f, charm_err *err)
{
    if (nmax > shc_nmax)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "\"nmax\" cannot be larger than \"shc_nmax\".");
        return;
    }
    if (kgrad < 0 || kgrad > 2 || (kgrad == 0 && dr + dlat + dlon > 2))
    {
        SET_ERR(err, CHARM_EFUNCARG, "Unsupported derivative selection.");
        return;
    }
    if (!check_type_shs(pnt, err))
        return;
    if (pnt->npoint == 0)
        return;
    report(err, __func__,
           cb::shs_point_dev(pnt, shc_nmax, mu, r, d_c, d_s, nmax, kgrad,
                             kgrad ? kgrad : (int)dr,
                             kgrad ? kgrad : (int)dlat,
                             kgrad ? kgrad : (int)dlon, d_f));
}

unsigned long charm_b200_shc_read_bin_dev(const char *pathname,
                                          unsigned long nmax,
                                          unsigned long shc_nmax, double *d_c,
                                          double *d_s, double *mu, double *r,
                                          charm_err *err)
{
    unsigned long nmax_file = CHARM_SHC_NMAX_ERROR;
    cb::Status st = cb::shc_read_bin_dev(pathname, nmax, shc_nmax, d_c, d_s,
                                         mu, r, &nmax_file);
    report(err, __func__, st);
    return st.ok() ? nmax_file : CHARM_SHC_NMAX_ERROR;
}

void charm_b200_shs_cell_dev(const charm_cell *cell, unsigned long shc_nmax,
                             double mu, double r, const double *d_c,
                             const double *d_s, unsigned long nmax,
                             double *d_f, charm_err *err)
{
    if (nmax > shc_nmax)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "\"nmax\" cannot be larger than \"shc_nmax\".");
        return;
    }
    if (cell->ncell == 0)
        return;
    if (!check_type_shs_cell(cell, err))
        return;
    report(err, __func__,
           cb::shs_cell_dev(cell, shc_nmax, mu, r, d_c, d_s, nmax, d_f));
}

void charm_b200_sha_cell_dev(const charm_cell *cell, const double *d_f,
                             unsigned long nmax, double mu, double r,
                             unsigned long shc_nmax, double *d_c,
                             double *d_s, charm_err *err)
{
    if (!check_sha_cell(cell, CHARM_SHA_CELL_AQ, err))
        return;
    if (nmax > shc_nmax)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "\"nmax\" cannot be larger than \"shc_nmax\".");
        return;
    }
    if (cell->ncell == 0)
        return;
    report(err, __func__,
           cb::sha_cell_dev(cell, d_f, nmax, mu, r, shc_nmax, d_c, d_s));
}

void charm_b200_sha_point_dev(const charm_point *pnt, const double *d_f,
                              unsigned long nmax, double mu, double r,
                              unsigned long shc_nmax, double *d_c,
                              double *d_s, charm_err *err)
{
    if (nmax > shc_nmax)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "\"nmax\" cannot be larger than \"shc_nmax\".");
        return;
    }
    if (!is_quad_type(pnt->type))
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "Unsupported \"pnt->type\" for spherical harmonic analysis of "
                "point data values.");
        return;
    }
    unsigned long nmax_grd = pnt->type == CHARM_CRD_POINT_GRID_GL
                                 ? (unsigned long)pnt->nlat - 1
                                 : ((unsigned long)pnt->nlat - 2) / 2;
    if (nmax > nmax_grd)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "The input data grid \"pnt\" was created for a maximum degree "
                "that is not high enough to recover harmonics up to the "
                "specified maximum degree of the analysis.");
        return;
    }
    report(err, __func__,
           cb::sha_point_dev(pnt, d_f, nmax, mu, r, shc_nmax, d_c, d_s));
}

// Batched synthesis: no CHarm counterpart (CHarm synthesises one set per
// call); each set gets the checks of charm_shs_point.
void charm_b200_shs_point_batch_dev(const charm_point *pnt, size_t nsets,
                                    const unsigned long *nmax,
                                    const unsigned long *shc_nmax,
                                    const double *mu, double r,
                                    const double *const *d_c,
                                    const double *const *d_s, int kgrad,
                                    double *const *d_f, charm_err *err)
{
    if (kgrad < 0 || kgrad > 3)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "\"kgrad\" must be 0 (potential), 1 (grad1), 2 (grad2) or "
                "3 (all ten quantities).");
        return;
    }
    if (!(pnt->type == CHARM_CRD_POINT_GRID ||
          is_quad_type(pnt->type)))
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "The batched synthesis works on grids (\"pnt->type\").");
        return;
    }
    for (size_t j = 0; j < nsets; j++)
        if (nmax[j] > shc_nmax[j])
        {
            char msg[CHARM_ERR_MAX_MSG];
            snprintf(msg, sizeof msg,
                     "Set %zu: \"nmax = %lu\" cannot be larger than the "
                     "degree of its coefficients \"%lu\".",
                     j, nmax[j], shc_nmax[j]);
            SET_ERR(err, CHARM_EFUNCARG, msg);
            return;
        }
    if (nsets == 0 || pnt->npoint == 0)
        return;
    report(err, __func__,
           cb::shs_point_batch_dev(pnt, nsets, nmax, shc_nmax, mu, r, d_c,
                                   d_s, kgrad, d_f));
}

// A batched synthesis captured into a CUDA graph (no CHarm counterpart):
// the checks of the batched entry points, then one plain call and the
// captured one.
void *charm_b200_shs_point_batch_graph(const charm_point *pnt, size_t nsets,
                                       const unsigned long *nmax,
                                       const unsigned long *shc_nmax,
                                       const double *mu, double r,
                                       const double *const *d_c,
                                       const double *const *d_s, int kgrad,
                                       double *const *d_f,
                                       int split_precision, charm_err *err)
{
    if (kgrad < 0 || kgrad > 3)
    {
        SET_ERR(err, CHARM_EFUNCARG, "\"kgrad\" must be 0..3.");
        return nullptr;
    }
    if (!(pnt->type == CHARM_CRD_POINT_GRID ||
          is_quad_type(pnt->type)))
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "The batched synthesis works on grids (\"pnt->type\").");
        return nullptr;
    }
    for (size_t j = 0; j < nsets; j++)
        if (nmax[j] > shc_nmax[j])
        {
            char msg[CHARM_ERR_MAX_MSG];
            snprintf(msg, sizeof msg,
                     "Set %zu: \"nmax = %lu\" cannot be larger than the "
                     "degree of its coefficients \"%lu\".",
                     j, nmax[j], shc_nmax[j]);
            SET_ERR(err, CHARM_EFUNCARG, msg);
            return nullptr;
        }
    if (nsets == 0 || pnt->npoint == 0)
    {
        SET_ERR(err, CHARM_EFUNCARG, "Nothing to capture (no sets or points).");
        return nullptr;
    }
    void *g = nullptr;
    report(err, __func__,
           cb::batch_graph_create(pnt, nsets, nmax, shc_nmax, mu, r, d_c, d_s,
                                  kgrad, d_f, split_precision, &g));
    return g;
}

void charm_b200_graph_launch(void *graph, charm_err *err)
{
    if (!graph)
    {
        SET_ERR(err, CHARM_EFUNCARG, "\"graph\" is NULL.");
        return;
    }
    report(err, __func__, cb::batch_graph_launch(graph));
}

void charm_b200_graph_free(void *graph)
{
    cb::batch_graph_free(graph);
}

// The synthesis autotuner's choices: copies up to n - 1 characters of the
// report (one line per problem shape: kernel, shape, chosen K and the
// measured milliseconds of every candidate) into buf; returns the full
// length.
size_t charm_b200_autotune_report(char *buf, size_t n)
{
    const std::string r = cb::autotune_report();
    if (buf && n > 0)
    {
        const size_t k = std::min(n - 1, r.size());
        std::memcpy(buf, r.data(), k);
        buf[k] = '\0';
    }
    return r.size();
}

// Split-precision batched synthesis: the same call with the degree sums on
// the tensor cores, kgrad 0..3 as the FP64 batch.
void charm_b200_shs_point_batch_i8_dev(const charm_point *pnt, size_t nsets,
                                       const unsigned long *nmax,
                                       const unsigned long *shc_nmax,
                                       const double *mu, double r,
                                       const double *const *d_c,
                                       const double *const *d_s, int kgrad,
                                       double *const *d_f, charm_err *err)
{
    if (kgrad < 0 || kgrad > 3)
    {
        SET_ERR(err, CHARM_EFUNCARG, "\"kgrad\" must be 0, 1, 2 or 3.");
        return;
    }
    if (!(pnt->type == CHARM_CRD_POINT_GRID ||
          is_quad_type(pnt->type)))
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "The batched synthesis works on grids (\"pnt->type\").");
        return;
    }
    for (size_t j = 0; j < nsets; j++)
        if (nmax[j] > shc_nmax[j])
        {
            char msg[CHARM_ERR_MAX_MSG];
            snprintf(msg, sizeof msg,
                     "Set %zu: \"nmax = %lu\" cannot be larger than the "
                     "degree of its coefficients \"%lu\".",
                     j, nmax[j], shc_nmax[j]);
            SET_ERR(err, CHARM_EFUNCARG, msg);
            return;
        }
    if (nsets == 0 || pnt->npoint == 0)
        return;
    report(err, __func__,
           cb::shs_point_batch_i8_dev(pnt, nsets, nmax, shc_nmax, mu, r, d_c,
                                      d_s, kgrad, d_f));
}

// Single-precision mode: no CHarm counterpart at this ABI level (CHarm's
// float build is a separate library, charmf_*); the checks mirror the
// double-precision device entry points.
void charm_b200_shs_point_dev_f32(const charm_point *pnt,
                                  unsigned long shc_nmax, double mu, double r,
                                  const float *d_c, const float *d_s,
                                  unsigned long nmax, float *d_f,
                                  charm_err *err)
{
    if (nmax > shc_nmax)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "\"nmax\" cannot be larger than \"shc_nmax\".");
        return;
    }
    if (pnt->type == CHARM_CRD_POINT_SCATTERED)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "The single-precision mode synthesises on grids only.");
        return;
    }
    if (pnt->npoint == 0)
        return;
    report(err, __func__,
           cb::shs_point_dev_f32(pnt, shc_nmax, mu, r, d_c, d_s, nmax, d_f));
}

void charm_b200_sha_point_dev_f32(const charm_point *pnt, const float *d_f,
                                  unsigned long nmax, double mu, double r,
                                  unsigned long shc_nmax, float *d_c,
                                  float *d_s, charm_err *err)
{
    if (nmax > shc_nmax)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "\"nmax\" cannot be larger than \"shc_nmax\".");
        return;
    }
    if (!is_quad_type(pnt->type))
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "Unsupported \"pnt->type\" for spherical harmonic analysis of "
                "point data values.");
        return;
    }
    unsigned long nmax_grd = pnt->type == CHARM_CRD_POINT_GRID_GL
                                 ? (unsigned long)pnt->nlat - 1
                                 : ((unsigned long)pnt->nlat - 2) / 2;
    if (nmax > nmax_grd)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "The input data grid \"pnt\" was created for a maximum degree "
                "that is not high enough to recover harmonics up to the "
                "specified maximum degree of the analysis.");
        return;
    }
    report(err, __func__,
           cb::sha_point_dev_f32(pnt, d_f, nmax, mu, r, shc_nmax, d_c, d_s));
}

// Adjoint of the scattered synthesis: no CHarm counterpart; the checks are
// those of charm_shs_point plus the point type.
static bool check_adjoint(const charm_point *pnt, unsigned long nmax,
                          unsigned long shc_nmax, charm_err *err)
{
    if (nmax > shc_nmax)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "\"nmax\" cannot be larger than the maximum harmonic degree "
                "of the coefficients.");
        return false;
    }
    if (pnt->type != CHARM_CRD_POINT_SCATTERED)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "The adjoint of the synthesis requires scattered points "
                "(\"pnt->type\" must be CHARM_CRD_POINT_SCATTERED).");
        return false;
    }
    return true;
}

void charm_b200_shs_point_sctr_adjoint(const charm_point *pnt,
                                       const double *g, unsigned long nmax,
                                       charm_shc *shcs, charm_err *err)
{
    if (!check_adjoint(pnt, nmax, shcs->nmax, err))
        return;
    if (pnt->npoint == 0)
    {
        // no points: every derivative is zero
        for (unsigned long m = 0; m <= shcs->nmax; m++)
            for (unsigned long n = m; n <= shcs->nmax; n++)
            {
                shcs->c[m][n - m] = 0.0;
                shcs->s[m][n - m] = 0.0;
            }
        return;
    }
    report(err, __func__, cb::shs_point_sctr_adjoint(pnt, g, nmax, shcs));
}

void charm_b200_shs_point_sctr_adjoint_dev(const charm_point *pnt,
                                           const double *d_g,
                                           unsigned long nmax, double mu,
                                           double r, unsigned long shc_nmax,
                                           double *d_c, double *d_s,
                                           charm_err *err)
{
    if (!check_adjoint(pnt, nmax, shc_nmax, err))
        return;
    if (pnt->npoint == 0)
    {
        const size_t T = (size_t)(shc_nmax + 1) * (shc_nmax + 2) / 2;
        cudaStream_t st = (cudaStream_t)cb::stream_handle();
        cudaMemsetAsync(d_c, 0, T * sizeof(double), st);
        cudaMemsetAsync(d_s, 0, T * sizeof(double), st);
        cudaStreamSynchronize(st);
        return;
    }
    report(err, __func__,
           cb::shs_point_sctr_adjoint_dev(pnt, d_g, nmax, mu, r, shc_nmax,
                                          d_c, d_s));
}

void charm_b200_sha_point_dev_static(const charm_point *pnt,
                                     const double *d_f, unsigned long nmax,
                                     double mu, double r,
                                     unsigned long shc_nmax, double *d_c,
                                     double *d_s, charm_err *err)
{
    if (nmax > shc_nmax)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "\"nmax\" cannot be larger than \"shc_nmax\".");
        return;
    }
    if (!is_quad_type(pnt->type))
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "Unsupported \"pnt->type\" for spherical harmonic analysis of "
                "point data values.");
        return;
    }
    unsigned long nmax_grd = pnt->type == CHARM_CRD_POINT_GRID_GL
                                 ? (unsigned long)pnt->nlat - 1
                                 : ((unsigned long)pnt->nlat - 2) / 2;
    if (nmax > nmax_grd)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "The input data grid \"pnt\" was created for a maximum degree "
                "that is not high enough to recover harmonics up to the "
                "specified maximum degree of the analysis.");
        return;
    }
    report(err, __func__,
           cb::sha_point_dev_static(pnt, d_f, nmax, mu, r, shc_nmax, d_c,
                                    d_s));
}

// Latitude-band analysis of a sharded transform: no CHarm counterpart (the
// reference's MPI build distributes latitude chunks, src/mpi, and reduces
// the coefficients, src/shc/shc_block_set_coeffs.c:80-86); the checks are
// charm_b200_sha_point_dev's.
void charm_b200_sha_point_dev_band(const charm_point *pnt, const double *d_f,
                                   unsigned long nmax, double mu, double r,
                                   unsigned long shc_nmax, int pair0,
                                   int pair1, double *d_c, double *d_s,
                                   charm_err *err)
{
    if (nmax > shc_nmax)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "\"nmax\" cannot be larger than \"shc_nmax\".");
        return;
    }
    if (!is_quad_type(pnt->type))
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "Unsupported \"pnt->type\" for spherical harmonic analysis of "
                "point data values.");
        return;
    }
    unsigned long nmax_grd = pnt->type == CHARM_CRD_POINT_GRID_GL
                                 ? (unsigned long)pnt->nlat - 1
                                 : ((unsigned long)pnt->nlat - 2) / 2;
    if (nmax > nmax_grd)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "The input data grid \"pnt\" was created for a maximum degree "
                "that is not high enough to recover harmonics up to the "
                "specified maximum degree of the analysis.");
        return;
    }
    report(err, __func__,
           cb::sha_point_dev_band(pnt, d_f, nmax, mu, r, shc_nmax, pair0,
                                  pair1, d_c, d_s));
}

int charm_b200_grid_pairs(const charm_point *pnt, int *row_n, int *row_s,
                          int cap)
{
    if (!pnt || !is_grid_type(pnt->type))
        return 0;
    return cb::grid_pair_rows(pnt, row_n, row_s, cap);
}

void *charm_b200_stream(void)
{
    return cb::stream_handle();
}

void charm_b200_timing(int enable)
{
    cb::set_timing(enable != 0);
}

int charm_b200_timing_read(double *ms, unsigned long long *count, int n,
                           unsigned long long *kernel_launches,
                           unsigned long long *fft_execs)
{
    double tms[cb::TIMER_COUNT];
    unsigned long long tn[cb::TIMER_COUNT];
    cb::read_timing(tms, tn, kernel_launches, fft_execs);
    for (int i = 0; i < n && i < cb::TIMER_COUNT; i++)
    {
        if (ms)
            ms[i] = tms[i];
        if (count)
            count[i] = tn[i];
    }
    return cb::TIMER_COUNT;
}

double charm_b200_fp64_peak_tflops(void)
{
    double t = -1.0;
    if (!cb::fp64_peak(&t).ok())
        return -1.0;
    return t;
}

} // extern "C"

// ---------------------------------------------------------------------------
// Single-precision ABI: CHarm's float build exports the same entry points
// with the prefix charmf_ and float arrays (src/prec.h:84-86 with @P@ = f;
// src/shs/shs.h.in:168-173, 239-244, 344-349, 428-435;
// src/sha/sha.h.in:164-169; src/crd/crd.h.in:477-760;
// src/shc/shc.h.in:423-602; src/err/err.h.in:236-294; src/glob/glob.c).
// Argument checks restate the double-precision ones above.  The transforms
// run on the single-precision kernels where they serve the call (potential
// on grids with FFT longitudes, nmax <= 2200, every row at the
// coefficients' radius), otherwise on the FP64 path with the results
// rounded to float.  Float inputs convert to double exactly; during a call
// the comparison thresholds are the float build's (charmf_glob_threshold*),
// as CHarm's float build applies them.
// ---------------------------------------------------------------------------
#include <vector>

extern "C"
{

CHARM_EXTERN float charmf_glob_threshold = 100.0f * FLT_EPSILON;
CHARM_EXTERN float charmf_glob_threshold2 = 100000.0f * FLT_EPSILON;
CHARM_EXTERN unsigned long charmf_glob_polar_optimization_a1 = 100;
CHARM_EXTERN float charmf_glob_polar_optimization_a2 = -1.0f;

charmf_err *charmf_err_init(void) { return charm_err_init(); }
void charmf_err_free(charmf_err *err) { charm_err_free(err); }
void charmf_err_reset(charmf_err *err) { charm_err_reset(err); }
void charmf_err_handler(charmf_err *err, _Bool terminate)
{
    charm_err_handler(err, terminate);
}
_Bool charmf_err_isempty(const charmf_err *err)
{
    return charm_err_isempty(err);
}

charmf_point *charmf_crd_point_init(int type, size_t nlat, size_t nlon,
                                    float *lat, float *lon, float *r)
{
    if (!is_point_type(type))
        return NULL;
    if (type == CHARM_CRD_POINT_SCATTERED && nlat != nlon)
        return NULL;
    charmf_point *p = (charmf_point *)malloc(sizeof(charmf_point));
    if (!p)
        return NULL;
    p->lat = p->lon = p->r = p->w = NULL;
    if (nlat > 0)
    {
        p->lat = lat;
        p->r = r;
    }
    if (nlon > 0)
        p->lon = lon;
    p->nlat = nlat;
    p->nlon = nlon;
    p->npoint = type == CHARM_CRD_POINT_SCATTERED ? nlat
                                                  : (is_grid_type(type)
                                                         ? nlat * nlon
                                                         : 0);
    p->type = type;
    p->owner = 0;
    p->distributed = 0;
    return p;
}

static charmf_point *pointf_alloc(int type, size_t nlat, size_t nlon,
                                  bool zero)
{
    if (!is_point_type(type))
        return NULL;
    if (type == CHARM_CRD_POINT_SCATTERED && nlat != nlon)
        return NULL;
    float *lat = NULL, *lon = NULL, *r = NULL, *w = NULL;
    auto al = [&](size_t n) -> float * {
        return zero ? (float *)calloc(n, sizeof(float))
                    : (float *)malloc(n * sizeof(float));
    };
    charmf_point *p = NULL;
    if (nlat > 0)
    {
        lat = al(nlat);
        r = al(nlat);
        if (!lat || !r)
            goto FAIL;
    }
    if (nlon > 0)
    {
        lon = al(nlon);
        if (!lon)
            goto FAIL;
    }
    p = charmf_crd_point_init(type, nlat, nlon, lat, lon, r);
    if (!p)
        goto FAIL;
    if (is_quad_type(type))
    {
        w = al(nlat > 0 ? nlat : 1);
        if (!w)
            goto FAIL;
        p->w = w;
    }
    p->owner = 1;
    return p;
FAIL:
    free(lat);
    free(lon);
    free(r);
    free(w);
    free(p);
    return NULL;
}

charmf_point *charmf_crd_point_malloc(int type, size_t nlat, size_t nlon)
{
    return pointf_alloc(type, nlat, nlon, false);
}

charmf_point *charmf_crd_point_calloc(int type, size_t nlat, size_t nlon)
{
    return pointf_alloc(type, nlat, nlon, true);
}

void charmf_crd_point_free(charmf_point *pnt)
{
    if (!pnt)
        return;
    if (pnt->owner)
    {
        free(pnt->lat);
        free(pnt->lon);
        free(pnt->r);
        free(pnt->w);
    }
    free(pnt);
}

void charmf_crd_point_gl_shape(unsigned long nmax, size_t *nlat, size_t *nlon)
{
    charm_crd_point_gl_shape(nmax, nlat, nlon);
}

void charmf_crd_point_dh1_shape(unsigned long nmax, size_t *nlat,
                                size_t *nlon)
{
    charm_crd_point_dh1_shape(nmax, nlat, nlon);
}

void charmf_crd_point_dh2_shape(unsigned long nmax, size_t *nlat,
                                size_t *nlon)
{
    charm_crd_point_dh2_shape(nmax, nlat, nlon);
}

// the double-precision grid (nodes from the GPU Newton iteration), rounded
static charmf_point *quad_gridf(int type, unsigned long nmax, float r)
{
    charm_point *d = quad_grid(type, nmax, (double)r);
    if (!d)
        return NULL;
    charmf_point *p = pointf_alloc(type, d->nlat, d->nlon, false);
    if (p)
    {
        for (size_t i = 0; i < d->nlat; i++)
        {
            p->lat[i] = (float)d->lat[i];
            p->r[i] = r;
            p->w[i] = (float)d->w[i];
        }
        for (size_t j = 0; j < d->nlon; j++)
            p->lon[j] = (float)d->lon[j];
    }
    charm_crd_point_free(d);
    return p;
}

charmf_point *charmf_crd_point_gl(unsigned long nmax, float r)
{
    return quad_gridf(CHARM_CRD_POINT_GRID_GL, nmax, r);
}

charmf_point *charmf_crd_point_dh1(unsigned long nmax, float r)
{
    return quad_gridf(CHARM_CRD_POINT_GRID_DH1, nmax, r);
}

charmf_point *charmf_crd_point_dh2(unsigned long nmax, float r)
{
    return quad_gridf(CHARM_CRD_POINT_GRID_DH2, nmax, r);
}

charmf_shc *charmf_shc_init(unsigned long nmax, float mu, float r, float *c,
                            float *s)
{
    if (r <= 0.0f)
        return NULL;
    charmf_shc *h = (charmf_shc *)malloc(sizeof(charmf_shc));
    if (!h)
        return NULL;
    h->nmax = nmax;
    h->mu = mu;
    h->r = r;
    size_t nmax1 = (size_t)nmax + 1;
    size_t len = ((nmax1 + 1) * nmax1) / 2;
    h->nc = h->ns = len;
    h->owner = 0;
    h->distributed = 0;
    h->c = (float **)malloc(nmax1 * sizeof(float *));
    h->s = (float **)malloc(nmax1 * sizeof(float *));
    if (!h->c || !h->s)
    {
        free(h->c);
        free(h->s);
        free(h);
        return NULL;
    }
    size_t idx = 0;
    for (size_t m = 0; m <= nmax; m++)
    {
        h->c[m] = c + idx;
        h->s[m] = s + idx;
        idx += nmax1 - m;
    }
    return h;
}

static charmf_shc *shcf_alloc(unsigned long nmax, float mu, float r,
                              bool zero)
{
    size_t nmax1 = (size_t)nmax + 1;
    size_t len = ((nmax1 + 1) * nmax1) / 2;
    float *c = zero ? (float *)calloc(len, sizeof(float))
                    : (float *)malloc(len * sizeof(float));
    float *s = zero ? (float *)calloc(len, sizeof(float))
                    : (float *)malloc(len * sizeof(float));
    charmf_shc *h = NULL;
    if (!c || !s)
        goto FAIL;
    h = charmf_shc_init(nmax, mu, r, c, s);
    if (!h)
        goto FAIL;
    h->owner = 1;
    return h;
FAIL:
    free(c);
    free(s);
    return NULL;
}

charmf_shc *charmf_shc_malloc(unsigned long nmax, float mu, float r)
{
    return shcf_alloc(nmax, mu, r, false);
}

charmf_shc *charmf_shc_calloc(unsigned long nmax, float mu, float r)
{
    return shcf_alloc(nmax, mu, r, true);
}

void charmf_shc_free(charmf_shc *shcs)
{
    if (!shcs)
        return;
    if (shcs->owner && shcs->c && shcs->s)
    {
        free(shcs->c[0]);
        free(shcs->s[0]);
    }
    free(shcs->c);
    free(shcs->s);
    free(shcs);
}

} // extern "C"

namespace
{

// the float build's thresholds in force for the duration of a call
struct FloatThresholds
{
    double t1, t2, a2;
    unsigned long a1;
    FloatThresholds()
        : t1(charm_glob_threshold), t2(charm_glob_threshold2),
          a2(charm_glob_polar_optimization_a2),
          a1(charm_glob_polar_optimization_a1)
    {
        charm_glob_threshold = (double)charmf_glob_threshold;
        charm_glob_threshold2 = (double)charmf_glob_threshold2;
        charm_glob_polar_optimization_a1 = charmf_glob_polar_optimization_a1;
        charm_glob_polar_optimization_a2 =
            (double)charmf_glob_polar_optimization_a2;
    }
    ~FloatThresholds()
    {
        charm_glob_threshold = t1;
        charm_glob_threshold2 = t2;
        charm_glob_polar_optimization_a1 = a1;
        charm_glob_polar_optimization_a2 = a2;
    }
};

// a charm_point over double copies of a charmf_point's arrays
struct PointD
{
    charm_point p{};
    std::vector<double> lat, lon, r, w;
    explicit PointD(const charmf_point *f)
    {
        auto cp = [](const float *src, size_t n, std::vector<double> &dst) {
            if (src)
                dst.assign(src, src + n);
        };
        cp(f->lat, f->nlat, lat);
        cp(f->lon, f->nlon, lon);
        cp(f->r, f->nlat, r);
        cp(f->w, f->nlat, w);
        p.type = f->type;
        p.nlat = f->nlat;
        p.nlon = f->nlon;
        p.npoint = f->npoint;
        p.lat = lat.empty() ? nullptr : lat.data();
        p.lon = lon.empty() ? nullptr : lon.data();
        p.r = r.empty() ? nullptr : r.data();
        p.w = w.empty() ? nullptr : w.data();
        p.owner = 0;
        p.distributed = 0;
    }
};

// a charm_shc over a contiguous double copy of a charmf_shc's triangle
struct ShcD
{
    charm_shc h{};
    std::vector<double> c, s;
    std::vector<double *> cp, sp;
    explicit ShcD(const charmf_shc *f, bool copy = true)
    {
        const size_t n1 = (size_t)f->nmax + 1;
        c.assign(n1 * (n1 + 1) / 2, 0.0);
        s.assign(c.size(), 0.0);
        cp.resize(n1);
        sp.resize(n1);
        size_t idx = 0;
        for (size_t m = 0; m < n1; m++)
        {
            if (copy)
                for (size_t k = 0; k < n1 - m; k++)
                {
                    c[idx + k] = (double)f->c[m][k];
                    s[idx + k] = (double)f->s[m][k];
                }
            cp[m] = c.data() + idx;
            sp[m] = s.data() + idx;
            idx += n1 - m;
        }
        h.nmax = f->nmax;
        h.mu = (double)f->mu;
        h.r = (double)f->r;
        h.nc = h.ns = c.size();
        h.c = cp.data();
        h.s = sp.data();
        h.owner = 0;
        h.distributed = 0;
    }
};

// contiguous float copy of a charmf_shc's triangle
void gather_tri(const charmf_shc *f, std::vector<float> &c,
                std::vector<float> &s)
{
    const size_t n1 = (size_t)f->nmax + 1;
    c.resize(n1 * (n1 + 1) / 2);
    s.resize(c.size());
    size_t idx = 0;
    for (size_t m = 0; m < n1; m++)
    {
        std::memcpy(c.data() + idx, f->c[m], (n1 - m) * sizeof(float));
        std::memcpy(s.data() + idx, f->s[m], (n1 - m) * sizeof(float));
        idx += n1 - m;
    }
}

bool check_nmax_f(const charmf_shc *shcs, unsigned long nmax, charm_err *err,
                  const char *what, const char *func)
{
    if (nmax > shcs->nmax)
    {
        char msg[CHARM_ERR_MAX_MSG];
        snprintf(msg, sizeof msg,
                 "Maximum harmonic degree of the %s \"nmax = %lu\" cannot be "
                 "larger than maximum harmonic degree of spherical harmonic "
                 "coefficients \"shcs->nmax = %lu\".",
                 what, nmax, shcs->nmax);
        err_set(err, __FILE__, __LINE__, func, CHARM_EFUNCARG, msg);
        return false;
    }
    return true;
}

// synthesis of npar components on the FP64 path, rounded into f[q]
void shs_f_fp64(const charmf_point *pnt, const charmf_shc *shcs,
                unsigned long nmax, int kgrad, int dr, int dlat, int dlon,
                int npar, float **f, charm_err *err, const char *func)
{
    PointD dp(pnt);
    ShcD dh(shcs);
    std::vector<std::vector<double>> out(npar,
                                         std::vector<double>(pnt->npoint));
    std::vector<double *> fp(npar);
    for (int q = 0; q < npar; q++)
        fp[q] = out[q].data();
    cb::Status st = cb::shs_point(&dp.p, &dh.h, nmax, kgrad, dr, dlat, dlon,
                                  fp.data());
    if (!st.ok())
    {
        err_set(err, __FILE__, __LINE__, func, st.code, st.msg.c_str());
        return;
    }
    for (int q = 0; q < npar; q++)
        for (size_t i = 0; i < pnt->npoint; i++)
            f[q][i] = (float)out[q][i];
}

bool check_type_shs_f(const charmf_point *pnt, charm_err *err,
                      const char *func)
{
    if (pnt->type != CHARM_CRD_POINT_SCATTERED && !is_grid_type(pnt->type))
    {
        err_set(err, __FILE__, __LINE__, func, CHARM_EFUNCARG,
                "Unsupported \"pnt->type\" for spherical harmonic synthesis "
                "of point values.");
        return false;
    }
    if (pnt->type == CHARM_CRD_POINT_SCATTERED && pnt->nlat != pnt->nlon)
    {
        err_set(err, __FILE__, __LINE__, func, CHARM_EFUNCARG,
                "The number of latitudes and longitudes in the \"pnt\" "
                "structure must be the same to perform point-wise spherical "
                "harmonic synthesis.");
        return false;
    }
    return true;
}

} // namespace

extern "C"
{

void charmf_shs_point(const charmf_point *pnt, const charmf_shc *shcs,
                      unsigned long nmax, float *f, charmf_err *err)
{
    if (!check_nmax_f(shcs, nmax, err, "synthesis", __func__))
        return;
    if (!check_type_shs_f(pnt, err, __func__))
        return;
    if (pnt->npoint == 0)
        return;
    FloatThresholds thr;
    PointD dp(pnt);
    if (cb::f32_serves(&dp.p, nmax, (double)shcs->r))
    {
        std::vector<float> c, s;
        gather_tri(shcs, c, s);
        report(err, __func__,
               cb::shs_point_f32_host(&dp.p, shcs->nmax, (double)shcs->mu,
                                      (double)shcs->r, c.data(), s.data(),
                                      nmax, f));
        return;
    }
    float *fp[1] = {f};
    shs_f_fp64(pnt, shcs, nmax, 0, 0, 0, 0, 1, fp, err, __func__);
}

void charmf_shs_point_grad1(const charmf_point *pnt, const charmf_shc *shcs,
                            unsigned long nmax, float **f, charmf_err *err)
{
    if (!check_nmax_f(shcs, nmax, err, "synthesis", __func__))
        return;
    if (!check_type_shs_f(pnt, err, __func__))
        return;
    if (pnt->npoint == 0)
        return;
    FloatThresholds thr;
    shs_f_fp64(pnt, shcs, nmax, 1, 1, 1, 1, 3, f, err, __func__);
    if (!charm_err_isempty(err))
        return;
    // src/shs/shs_point_gradn.c:133-145
    float *fx = f[2], *fy = f[0], *fz = f[1];
    f[0] = fx;
    f[1] = fy;
    f[2] = fz;
}

void charmf_shs_point_grad2(const charmf_point *pnt, const charmf_shc *shcs,
                            unsigned long nmax, float **f, charmf_err *err)
{
    if (!check_nmax_f(shcs, nmax, err, "synthesis", __func__))
        return;
    if (!check_type_shs_f(pnt, err, __func__))
        return;
    if (pnt->npoint == 0)
        return;
    FloatThresholds thr;
    shs_f_fp64(pnt, shcs, nmax, 2, 2, 2, 2, 6, f, err, __func__);
    if (!charm_err_isempty(err))
        return;
    // src/shs/shs_point_gradn.c:146-165
    float *fxx = f[5], *fxy = f[2], *fxz = f[4];
    float *fyy = f[0], *fyz = f[1], *fzz = f[3];
    f[0] = fxx;
    f[1] = fxy;
    f[2] = fxz;
    f[3] = fyy;
    f[4] = fyz;
    f[5] = fzz;
}

void charmf_shs_point_guru(const charmf_point *pnt, const charmf_shc *shcs,
                           unsigned long nmax, unsigned dr, unsigned dlat,
                           unsigned dlon, float *f, charmf_err *err)
{
    if (!check_nmax_f(shcs, nmax, err, "synthesis", __func__))
        return;
    if ((int)dr < 0 || (int)dlat < 0 || (int)dlon < 0 || dr + dlat + dlon > 2)
    {
        char msg[CHARM_ERR_MAX_MSG];
        snprintf(msg, sizeof msg,
                 "The sum \"dr + dlat + dlon\" is \"%d\", but it cannot be "
                 "larger than \"%d\".",
                 (int)(dr + dlat + dlon), 2);
        SET_ERR(err, CHARM_EFUNCARG, msg);
        return;
    }
    if (pnt->npoint == 0)
        return;
    if (!check_type_shs_f(pnt, err, __func__))
        return;
    FloatThresholds thr;
    float *fp[1] = {f};
    shs_f_fp64(pnt, shcs, nmax, 0, (int)dr, (int)dlat, (int)dlon, 1, fp, err,
               __func__);
}

void charmf_sha_point(const charmf_point *pnt, const float *f,
                      unsigned long nmax, charmf_shc *shcs, charmf_err *err)
{
    if (!check_nmax_f(shcs, nmax, err, "analysis", __func__))
        return;
    if (!is_quad_type(pnt->type))
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "Unsupported \"pnt->type\" for spherical harmonic analysis of "
                "point data values.");
        return;
    }
    FloatThresholds thr;
    const double r0 = (double)pnt->r[0];
    for (size_t i = 1; i < pnt->nlat; i++)
    {
        if (!nearly_equal((double)pnt->r[i], r0, charm_glob_threshold))
        {
            SET_ERR(err, CHARM_EFUNCARG,
                    "All spherical radii in \"pnt->r\" must be equal.");
            return;
        }
    }
    unsigned long nmax_grd = pnt->type == CHARM_CRD_POINT_GRID_GL
                                 ? (unsigned long)pnt->nlat - 1
                                 : ((unsigned long)pnt->nlat - 2) / 2;
    if (nmax > nmax_grd)
    {
        SET_ERR(err, CHARM_EFUNCARG,
                "The input data grid \"pnt\" was created for a maximum degree "
                "that is not high enough to recover harmonics up to the "
                "specified maximum degree of the analysis.");
        return;
    }
    PointD dp(pnt);
    const size_t n1 = (size_t)shcs->nmax + 1;
    if (cb::f32_serves(&dp.p, nmax, (double)shcs->r))
    {
        std::vector<float> c(n1 * (n1 + 1) / 2, 0.0f), s(c.size(), 0.0f);
        cb::Status st = cb::sha_point_f32_host(
            &dp.p, f, nmax, (double)shcs->mu, (double)shcs->r, shcs->nmax,
            c.data(), s.data());
        report(err, __func__, st);
        if (!st.ok())
            return;
        size_t idx = 0;
        for (size_t m = 0; m < n1; m++)
        {
            for (size_t k = 0; k < n1 - m; k++)
            {
                const bool keep = m + k <= nmax;
                shcs->c[m][k] = keep ? c[idx + k] : 0.0f;
                shcs->s[m][k] = keep ? s[idx + k] : 0.0f;
            }
            idx += n1 - m;
        }
        return;
    }
    ShcD dh(shcs, false);
    std::vector<double> fd(f, f + pnt->npoint);
    cb::Status st = cb::sha_point(&dp.p, fd.data(), nmax, &dh.h);
    report(err, __func__, st);
    if (!st.ok())
        return;
    size_t idx = 0;
    for (size_t m = 0; m < n1; m++)
    {
        for (size_t k = 0; k < n1 - m; k++)
        {
            shcs->c[m][k] = (float)dh.c[idx + k];
            shcs->s[m][k] = (float)dh.s[idx + k];
        }
        idx += n1 - m;
    }
}

} // extern "C"
