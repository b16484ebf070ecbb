/* psst_oracle.c — CPU restatement of the PSST explicit finite-volume loop.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path (see psst_oracle.h).
 * Every arithmetic expression below keeps the reference's operand order and
 * association so that results agree bit for bit with the reference compiled
 * without FMA contraction (-ffp-contract=off). Citations are file:line in the
 * reference project.
 */
#define _GNU_SOURCE
#include "psst_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define MAXD 3
#define MAXV 5 /* dim + 2 */
#define NG 6   /* gradient variables: u.. (dim), p, T, rho */

typedef struct {
    long id, first, last, bc, size;
    char name[128];
} zone_t;

typedef struct {
    long id, bc, first_vol, count; /* volumes of this zone: [first_vol, first_vol+count) */
    int dyn, therm;                /* boundary condition ids from .bvp/.btq (0 = none) */
    double bc_u[MAXD], bc_p, bc_T;
    int zs;                        /* index in zones (file order) */
} vzone_t;

typedef struct {
    long id, bc, first_face, count;
    int zs;
} fzone_t;

struct oracle {
    char err[512];
    int dim;
    /* ---- file level (psstAnsysInputGrid) ---- */
    long nvert;
    double *vx;
    long nff;                /* faces_ (append order) */
    long *ff_ptr, *ff_nodes; /* 1-based vertex ids */
    long *ff_c0, *ff_c1, *ff_zone;
    long nfc; /* cells_ */
    long *fc_zone;
    long nz;
    zone_t *z; /* zones_storage_ in file order */
    /* ---- finite-volume grid ---- */
    long nvz, nfz;
    vzone_t *vz; /* map order */
    fzone_t *fz; /* map order */
    long nvol, nface;
    int *v_boundary;
    long *v_vz; /* volume -> vzone index */
    long *v_fcnt, *v_fcap, **v_f; /* per-volume face list (wiring order) */
    double *V, *xc;
    long *f_c0, *f_c1, *f_fz, *f_loc; /* volume indices (-1 = none), fzone, file face loc */
    double *S, *n, *xf, *beta;
    double min_vol;
    /* ---- state ---- */
    double *p, *T, *rho, *u, *w, *pw, *res, *dt, *g; /* g: nvol x NG x dim */
    double *u_old, *T_old;                            /* Jacobi snapshot */
    double *res_conv;                                 /* oracle_convective output */
    /* ---- scheme ---- */
    double M, cp, rm, gamma, cv, ref_vel, CFL;
    long iter, max_iter, iter_step;
    int lc, rk_level, flux, order, gradm, limiter, lc1_jacobi;
    double rk[64];
    double venkat_k;
    double *lsq_r; /* LSQ_NR coefficients per zone-local index (quirk of psstLeastSquare) */
    long lsq_n;
    double *lim; /* per volume x NG limiter value (BJ/VK extension) */
};

static int fail(oracle_t *o, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(o->err, sizeof o->err, fmt, ap);
    va_end(ap);
    return -1;
}

/* ------------------------------------------------------------------------ */
/* text stream mirroring the std::istream operations the reference uses      */
/* ------------------------------------------------------------------------ */
typedef struct {
    char *buf;
    long len, pos;
} strm_t;

static int load_file(const char *path, strm_t *s) {
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    s->buf = (char *)malloc(n + 1);
    long r = (long)fread(s->buf, 1, n, f);
    fclose(f);
    /* CRLF files make the reference's reader loop forever on Linux; the
     * restatement reads the same content with CR removed. */
    long m = 0;
    for (long i = 0; i < r; ++i)
        if (s->buf[i] != '\r') s->buf[m++] = s->buf[i];
    s->buf[m] = 0;
    s->len = m;
    s->pos = 0;
    return 0;
}
static int s_eof(strm_t *s) { return s->pos >= s->len; }
static void s_skipws(strm_t *s) {
    while (s->pos < s->len && (s->buf[s->pos] == ' ' || s->buf[s->pos] == '\t' || s->buf[s->pos] == '\n' ||
                               s->buf[s->pos] == '\v' || s->buf[s->pos] == '\f'))
        s->pos++;
}
/* operator>>(double&) */
static int s_double(strm_t *s, double *x) {
    s_skipws(s);
    if (s_eof(s)) return -1;
    char *end;
    double v = strtod(s->buf + s->pos, &end);
    if (end == s->buf + s->pos) return -1;
    s->pos = end - s->buf;
    *x = v;
    return 0;
}
/* operator>>(size_t&) in std::hex or decimal mode */
static int s_ulong(strm_t *s, long *x, int base) {
    s_skipws(s);
    if (s_eof(s)) return -1;
    char *end;
    long v = strtol(s->buf + s->pos, &end, base);
    if (end == s->buf + s->pos) return -1;
    s->pos = end - s->buf;
    *x = v;
    return 0;
}
static int s_word(strm_t *s, char *out, int cap) {
    s_skipws(s);
    if (s_eof(s)) return -1;
    int k = 0;
    while (s->pos < s->len && !(s->buf[s->pos] == ' ' || s->buf[s->pos] == '\t' || s->buf[s->pos] == '\n')) {
        if (k < cap - 1) out[k++] = s->buf[s->pos];
        s->pos++;
    }
    out[k] = 0;
    return 0;
}
/* get_parameter (psstFiniteVolumeGrid.cpp:20-27): a double, then the rest of the line */
static double get_parameter(strm_t *s) {
    double x = 0.0;
    s_double(s, &x);
    while (s->pos < s->len && s->buf[s->pos++] != '\n') continue;
    return x;
}
static void s_getline(strm_t *s, char **line, long *len) {
    long b = s->pos;
    while (s->pos < s->len && s->buf[s->pos] != '\n') s->pos++;
    *line = s->buf + b;
    *len = s->pos - b;
    if (s->pos < s->len) s->pos++;
}

/* ------------------------------------------------------------------------ */
/* Fluent ASCII reader (psstAnsysDirector::build_step, :1138-1306)           */
/* ------------------------------------------------------------------------ */
typedef struct {
    char *line;
    long len, pos;
} lineparse_t;

/* private_parse_number (:1319-1374) */
static long parse_number(lineparse_t *lp, int base) {
    char buf[64];
    int k = 0, empty = 1;
    long dest = 0;
    while (lp->pos < lp->len) {
        char c = lp->line[lp->pos];
        int digit = (c >= '0' && c <= '9') ||
                    (base == 16 && ((c >= 'a' && c <= 'f') || (c >= 'A' && c <= 'F')));
        if (digit) {
            if (k < 63) buf[k++] = c;
            empty = 0;
        } else if (c == ' ' || c == '(' || c == ')') {
            if (!empty) {
                buf[k] = 0;
                dest = strtol(buf, NULL, base);
                break;
            }
        } else {
            break;
        }
        lp->pos++;
    }
    return dest;
}
/* private_parse_name (:1376-1398) */
static void parse_name(lineparse_t *lp, char *out, int cap) {
    int k = 0, empty = 1;
    while (lp->pos < lp->len) {
        char c = lp->line[lp->pos];
        if (c != ' ' && c != '(' && c != ')') {
            if (k < cap - 1) out[k++] = c;
            empty = 0;
        } else if (!empty) {
            break;
        }
        lp->pos++;
    }
    out[k] = 0;
}
/* the "header line does not end with '('" check repeated in build_step */
static void maybe_skip_line(lineparse_t *lp, strm_t *s) {
    for (long i = lp->len; i > 0; --i) {
        char ch = i < lp->len ? lp->line[i] : '\0';
        if (ch == ' ' || ch == '\0') continue;
        if (ch == '(') break;
        char *l;
        long n;
        s_getline(s, &l, &n);
        break;
    }
}
static long zone_find(oracle_t *o, long id) {
    for (long i = 0; i < o->nz; ++i)
        if (o->z[i].id == id) return i;
    return -1;
}
static long zone_add(oracle_t *o, long id) {
    long i = zone_find(o, id);
    if (i >= 0) return i;
    o->z = (zone_t *)realloc(o->z, sizeof(zone_t) * (o->nz + 1));
    memset(&o->z[o->nz], 0, sizeof(zone_t));
    o->z[o->nz].id = id;
    return o->nz++;
}

static int read_mesh(oracle_t *o, const char *path) {
    strm_t s;
    if (load_file(path, &s)) return fail(o, "Error: Could not open \"%s\" file!", path);
    long cap_ff = 0, cap_nodes = 0, cap_fc = 0, nnodes = 0;
    o->dim = 0;
    while (!s_eof(&s)) {
        char *l;
        long n;
        s_getline(&s, &l, &n);
        lineparse_t lp = {l, n, 0};
        long op = parse_number(&lp, 10);
        if (op == 2) {
            o->dim = (int)parse_number(&lp, 16);
        } else if (op == 10) {
            long zid = parse_number(&lp, 16), first = parse_number(&lp, 16), last = parse_number(&lp, 16);
            parse_number(&lp, 16);
            parse_number(&lp, 16);
            if (zid == 0) continue;
            maybe_skip_line(&lp, &s);
            long cnt = last - first + 1;
            o->vx = (double *)realloc(o->vx, sizeof(double) * (o->nvert + cnt) * o->dim);
            for (long i = 0; i < cnt; ++i)
                for (int j = 0; j < o->dim; ++j)
                    if (s_double(&s, &o->vx[(o->nvert + i) * o->dim + j]))
                        return fail(o, "mesh: truncated vertex section");
            o->nvert += cnt;
        } else if (op == 12) {
            long zid = parse_number(&lp, 16), first = parse_number(&lp, 16), last = parse_number(&lp, 16);
            long bc = parse_number(&lp, 16), type = parse_number(&lp, 16);
            if (zid == 0) continue;
            maybe_skip_line(&lp, &s);
            long zi = zone_add(o, zid);
            o->z[zi].first = first;
            o->z[zi].last = last;
            o->z[zi].bc = bc;
            o->z[zi].size = last - first + 1;
            long cnt = last - first + 1;
            if (o->nfc + cnt > cap_fc) {
                cap_fc = 2 * (o->nfc + cnt);
                o->fc_zone = (long *)realloc(o->fc_zone, sizeof(long) * cap_fc);
            }
            for (long i = 0; i < cnt; ++i) {
                long t = type;
                if (type == 0 && s_ulong(&s, &t, 16)) return fail(o, "mesh: truncated cell section");
                o->fc_zone[o->nfc++] = zid;
            }
        } else if (op == 13) {
            long zid = parse_number(&lp, 16), first = parse_number(&lp, 16), last = parse_number(&lp, 16);
            long bc = 0, ftype = 0;
            if (zid == 0) continue;
            bc = parse_number(&lp, 16);
            ftype = parse_number(&lp, 16);
            maybe_skip_line(&lp, &s);
            long zi = zone_add(o, zid);
            o->z[zi].first = first;
            o->z[zi].last = last;
            o->z[zi].bc = bc;
            o->z[zi].size = last - first + 1;
            long cnt = last - first + 1;
            if (o->nff + cnt + 1 > cap_ff) {
                cap_ff = 2 * (o->nff + cnt + 1);
                o->ff_ptr = (long *)realloc(o->ff_ptr, sizeof(long) * (cap_ff + 1));
                o->ff_c0 = (long *)realloc(o->ff_c0, sizeof(long) * cap_ff);
                o->ff_c1 = (long *)realloc(o->ff_c1, sizeof(long) * cap_ff);
                o->ff_zone = (long *)realloc(o->ff_zone, sizeof(long) * cap_ff);
            }
            if (o->nff == 0) o->ff_ptr[0] = 0;
            for (long i = 0; i < cnt; ++i) {
                long t = ftype;
                if (ftype == 0 && s_ulong(&s, &t, 16)) return fail(o, "mesh: truncated face section");
                long nv = (t == 2 || t == 3 || t == 4) ? t : -1;
                if (nv < 0) return fail(o, "Error: Unknown face type!");
                if (nnodes + nv > cap_nodes) {
                    cap_nodes = 2 * (nnodes + nv) + 16;
                    o->ff_nodes = (long *)realloc(o->ff_nodes, sizeof(long) * cap_nodes);
                }
                for (long j = 0; j < nv; ++j)
                    if (s_ulong(&s, &o->ff_nodes[nnodes + j], 16)) return fail(o, "mesh: truncated face");
                long c[2];
                if (s_ulong(&s, &c[0], 16) || s_ulong(&s, &c[1], 16)) return fail(o, "mesh: truncated face");
                nnodes += nv;
                /* read_faces passes (cells[1], cells[0]) as (left, right) and
                 * psstSimpleFace stores cell(0)=right, cell(1)=left
                 * (:1026, :192-193): file c0 stays neighbour 0. */
                o->ff_c0[o->nff] = c[0];
                o->ff_c1[o->nff] = c[1];
                o->ff_zone[o->nff] = zid;
                o->ff_ptr[o->nff + 1] = nnodes;
                o->nff++;
            }
        } else if (op == 39 || op == 45) {
            long zid = parse_number(&lp, 10);
            char tmp[128], name[128];
            parse_name(&lp, tmp, sizeof tmp);
            parse_name(&lp, name, sizeof name);
            long zi = zone_add(o, zid);
            snprintf(o->z[zi].name, sizeof o->z[zi].name, "%s", name);
        } else if (op == 58 || op == 59) {
            /* cell/face trees of adapted meshes (psstAnsysBuilder::read_cell_tree /
             * read_face_tree, psstAnsysGridReader.cpp:1068-1116): parent/child
             * links that no step of the loop reads; the parent zone gets bc 31
             * if no section declared it (add_zones_storage_connection, :655-686) */
            long first = parse_number(&lp, 16), last = parse_number(&lp, 16);
            long parent = parse_number(&lp, 16);
            (void)parse_number(&lp, 16);
            maybe_skip_line(&lp, &s);
            int known = 0;
            for (long zi = 0; zi < o->nz; ++zi)
                if (o->z[zi].id == parent) known = 1;
            if (!known) {
                long zi = zone_add(o, parent);
                o->z[zi].first = first;
                o->z[zi].last = last;
                o->z[zi].bc = 31;
                o->z[zi].size = last - first + 1;
            }
            for (long i = 0; i < last - first + 1; ++i) {
                long nk, kid;
                if (s_ulong(&s, &nk, 16)) return fail(o, "mesh: truncated tree section");
                for (long j = 0; j < nk; ++j)
                    if (s_ulong(&s, &kid, 16)) return fail(o, "mesh: truncated tree section");
            }
        }
    }
    free(s.buf);
    if (o->dim != 2 && o->dim != 3) return fail(o, "mesh: missing or invalid dimension section");
    return 0;
}

/* ------------------------------------------------------------------------ */
/* geometry: psstFace::initialize (:397-505), psstVolume::initialize (:709-827) */
/* ------------------------------------------------------------------------ */
static const double *vert(oracle_t *o, long id1) { return &o->vx[(id1 - 1) * o->dim]; }

static int face_init(oracle_t *o, long f) {
    long loc = o->f_loc[f];
    long nv = o->ff_ptr[loc + 1] - o->ff_ptr[loc];
    const long *nodes = &o->ff_nodes[o->ff_ptr[loc]];
    int dim = o->dim;
    double sq = 0.0, nn[3] = {0, 0, 0}, c[3] = {0, 0, 0};
    if (dim == 2) {
        if (nv != 2) return fail(o, "Error: Expected to vertices but extra data found!");
        const double *v0 = vert(o, nodes[0]), *v1 = vert(o, nodes[1]);
        for (int i = 0; i < 2; ++i) {
            c[i] = 0.5 * (v1[i] + v0[i]);
            double comp = v1[i] - v0[i];
            sq += comp * comp;
        }
        sq = sqrt(sq);
        nn[0] = v0[1] - v1[1];
        nn[1] = v1[0] - v0[0];
    } else {
        if (nv < 3) return fail(o, "Error: Expected at least 3 vertices!");
        double avg[3] = {0, 0, 0}, avg3[3] = {0, 0, 0};
        for (int i = 0; i < 3; ++i) {
            for (long j = 0; j < nv; ++j) avg[i] += vert(o, nodes[j])[i];
            avg[i] /= (double)nv;
            avg3[i] = avg[i] * 3;
        }
        double a[3], b[3], cc[3], ts;
        long last = nv - 1;
        for (long i = 0; i < last; ++i) {
            for (int j = 0; j < 3; ++j) {
                a[j] = vert(o, nodes[i])[j] - avg[j];
                b[j] = vert(o, nodes[i + 1])[j] - avg[j];
            }
            cc[0] = a[1] * b[2] - a[2] * b[1];
            cc[1] = a[2] * b[0] - a[0] * b[2];
            cc[2] = a[0] * b[1] - a[1] * b[0];
            ts = 0.0;
            for (int j = 0; j < 3; ++j) ts += cc[j] * cc[j];
            ts = sqrt(ts);
            sq += ts;
            for (int j = 0; j < 3; ++j) c[j] += ts * (a[j] + b[j] + avg3[j]);
        }
        for (int j = 0; j < 3; ++j) {
            a[j] = vert(o, nodes[last])[j] - avg[j];
            b[j] = vert(o, nodes[0])[j] - avg[j];
        }
        cc[0] = a[1] * b[2] - a[2] * b[1];
        cc[1] = a[2] * b[0] - a[0] * b[2];
        cc[2] = a[0] * b[1] - a[1] * b[0];
        ts = 0.0;
        for (int j = 0; j < 3; ++j) ts += cc[j] * cc[j];
        ts = sqrt(ts);
        sq += ts;
        double sq3 = sq * 3;
        for (int j = 0; j < 3; ++j) {
            c[j] += ts * (a[j] + b[j] + avg3[j]);
            c[j] /= sq3;
            nn[j] = cc[j];
        }
        sq *= 0.5;
    }
    /* psstGeometryVector::initialize + normalize (:248-256, :279-290) */
    double len = 0.0;
    for (int i = 0; i < dim; ++i) len += nn[i] * nn[i];
    len = sqrt(len);
    if (fabs(len) < 1.0e-10) return fail(o, "Error: Division by zero detected!");
    for (int i = 0; i < dim; ++i) nn[i] /= len;
    o->S[f] = sq;
    for (int i = 0; i < dim; ++i) {
        o->n[f * dim + i] = nn[i];
        o->xf[f * dim + i] = c[i];
    }
    return 0;
}

static long face_other(oracle_t *o, long f, long v) { return o->f_c0[f] == v ? o->f_c1[f] : o->f_c0[f]; }

static void volume_init(oracle_t *o, long v) {
    int dim = o->dim;
    long nf = o->v_fcnt[v];
    long *fl = o->v_f[v];
    double *x = &o->xc[v * dim];
    for (int i = 0; i < dim; ++i) x[i] = 0.0;
    o->V[v] = 0.0;
    if (o->v_boundary[v]) {
        for (int i = 0; i < dim; ++i) x[i] = o->xf[fl[0] * dim + i];
        return;
    }
    double vol = 0.0;
    if (dim == 2) {
        double avg[2] = {0, 0}, avg3[2] = {0, 0};
        for (int j = 0; j < 2; ++j) {
            for (long i = 0; i < nf; ++i) avg[j] += o->xf[fl[i] * 2 + j];
            avg[j] /= (double)nf;
            avg3[j] = avg[j] * 3;
        }
        for (long i = 0; i < nf; ++i) {
            long loc = o->f_loc[fl[i]];
            const long *nodes = &o->ff_nodes[o->ff_ptr[loc]];
            double a[2], b[2];
            for (int k = 0; k < 2; ++k) {
                a[k] = vert(o, nodes[0])[k] - avg[k];
                b[k] = vert(o, nodes[1])[k] - avg[k];
            }
            double tv = fabs(a[0] * b[1] - a[1] * b[0]);
            vol += tv;
            for (int k = 0; k < 2; ++k) x[k] += tv * (a[k] + b[k] + avg3[k]);
        }
        double v3 = vol * 3;
        for (int k = 0; k < 2; ++k) x[k] /= v3;
        vol /= 2;
    } else {
        double avg[3] = {0, 0, 0}, avg4[3] = {0, 0, 0};
        for (int j = 0; j < 3; ++j) {
            for (long i = 0; i < nf; ++i) avg[j] += o->xf[fl[i] * 3 + j];
            avg[j] /= (double)nf;
            avg4[j] = avg[j] * 4;
        }
        for (long i = 0; i < nf; ++i) {
            long loc = o->f_loc[fl[i]];
            long nv = o->ff_ptr[loc + 1] - o->ff_ptr[loc];
            const long *nodes = &o->ff_nodes[o->ff_ptr[loc]];
            const double *cen = &o->xf[fl[i] * 3];
            for (long j = 0; j < nv; ++j) {
                long nx = j + 1;
                if (nx == nv) nx = 0;
                double a[3], b[3], c[3];
                for (int k = 0; k < 3; ++k) {
                    a[k] = vert(o, nodes[j])[k] - avg[k];
                    b[k] = vert(o, nodes[nx])[k] - avg[k];
                    c[k] = cen[k] - avg[k];
                }
                double tv = fabs(a[0] * (b[1] * c[2] - b[2] * c[1]) - a[1] * (b[0] * c[2] - b[2] * c[0]) +
                                 a[2] * (b[0] * c[1] - b[1] * c[0]));
                vol += tv;
                for (int k = 0; k < 3; ++k) x[k] += tv * (a[k] + b[k] + c[k] + avg4[k]);
            }
        }
        double v4 = vol * 4.0;
        for (int k = 0; k < 3; ++k) x[k] /= v4;
        vol /= 6.0;
    }
    o->V[v] = vol;
}

static long vz_find(oracle_t *o, long id) {
    for (long i = 0; i < o->nvz; ++i)
        if (o->vz[i].id == id) return i;
    return -1;
}
static long fz_find(oracle_t *o, long id) {
    for (long i = 0; i < o->nfz; ++i)
        if (o->fz[i].id == id) return i;
    return -1;
}
static int cmp_zone_id(const void *a, const void *b) {
    long x = *(const long *)a, y = *(const long *)b;
    return x < y ? -1 : x > y;
}
static void vol_add_face(oracle_t *o, long v, long f) {
    if (o->v_fcnt[v] == o->v_fcap[v]) {
        o->v_fcap[v] = o->v_fcap[v] ? 2 * o->v_fcap[v] : 4;
        o->v_f[v] = (long *)realloc(o->v_f[v], sizeof(long) * o->v_fcap[v]);
    }
    o->v_f[v][o->v_fcnt[v]++] = f;
}

/* psstAnsysInputGrid::create_finite_volume_grid (:688-907) */
static int build_fv(oracle_t *o) {
    long *vids = (long *)malloc(sizeof(long) * (o->nz + 1));
    long *fids = (long *)malloc(sizeof(long) * (o->nz + 1));
    long nv = 0, nf = 0;
    for (long i = 0; i < o->nz; ++i) {
        long bc = o->z[i].bc;
        if (bc == 1 || bc == 32)
            vids[nv++] = o->z[i].id;
        else if (bc == 2 || bc == 31)
            fids[nf++] = o->z[i].id;
        else {
            vids[nv++] = o->z[i].id;
            fids[nf++] = o->z[i].id;
        }
    }
    qsort(vids, nv, sizeof(long), cmp_zone_id);
    qsort(fids, nf, sizeof(long), cmp_zone_id);
    o->nvz = nv;
    o->nfz = nf;
    o->vz = (vzone_t *)calloc(nv ? nv : 1, sizeof(vzone_t));
    o->fz = (fzone_t *)calloc(nf ? nf : 1, sizeof(fzone_t));
    long tv = 0, tf = 0;
    for (long i = 0; i < nv; ++i) {
        long zs = zone_find(o, vids[i]);
        o->vz[i].id = vids[i];
        o->vz[i].bc = o->z[zs].bc;
        o->vz[i].zs = (int)zs;
        o->vz[i].first_vol = tv;
        o->vz[i].count = o->z[zs].size;
        tv += o->z[zs].size;
    }
    for (long i = 0; i < nf; ++i) {
        long zs = zone_find(o, fids[i]);
        o->fz[i].id = fids[i];
        o->fz[i].bc = o->z[zs].bc;
        o->fz[i].zs = (int)zs;
        o->fz[i].first_face = tf;
        o->fz[i].count = o->z[zs].size;
        tf += o->z[zs].size;
    }
    free(vids);
    free(fids);
    o->nvol = tv;
    o->nface = tf;
    int dim = o->dim;
    o->v_boundary = (int *)calloc(tv + 1, sizeof(int));
    o->v_vz = (long *)calloc(tv + 1, sizeof(long));
    o->v_fcnt = (long *)calloc(tv + 1, sizeof(long));
    o->v_fcap = (long *)calloc(tv + 1, sizeof(long));
    o->v_f = (long **)calloc(tv + 1, sizeof(long *));
    o->V = (double *)calloc(tv + 1, sizeof(double));
    o->xc = (double *)calloc((tv + 1) * dim, sizeof(double));
    for (long i = 0; i < o->nvz; ++i) {
        int bnd = !(o->vz[i].bc == 1 || o->vz[i].bc == 32);
        for (long j = 0; j < o->vz[i].count; ++j) {
            o->v_boundary[o->vz[i].first_vol + j] = bnd;
            o->v_vz[o->vz[i].first_vol + j] = i;
        }
    }
    o->f_c0 = (long *)malloc(sizeof(long) * (tf + 1));
    o->f_c1 = (long *)malloc(sizeof(long) * (tf + 1));
    o->f_fz = (long *)malloc(sizeof(long) * (tf + 1));
    o->f_loc = (long *)malloc(sizeof(long) * (tf + 1));
    o->S = (double *)calloc(tf + 1, sizeof(double));
    o->n = (double *)calloc((tf + 1) * dim, sizeof(double));
    o->xf = (double *)calloc((tf + 1) * dim, sizeof(double));
    o->beta = (double *)calloc(tf + 1, sizeof(double));
    for (long i = 0; i < o->nfz; ++i)
        for (long j = 0; j < o->fz[i].count; ++j) {
            long f = o->fz[i].first_face + j;
            o->f_fz[f] = i;
            o->f_loc[f] = o->z[o->fz[i].zs].first + j - 1;
            o->f_c0[f] = o->f_c1[f] = -1;
            if (o->f_loc[f] < 0 || o->f_loc[f] >= o->nff) return fail(o, "mesh: face index out of range");
        }
    /* wiring, zones in file order (:825-883) */
    for (long zi = 0; zi < o->nz; ++zi) {
        long bc = o->z[zi].bc;
        if (bc == 1 || bc == 32) continue;
        long fzi = fz_find(o, o->z[zi].id);
        for (long j = 0; j < o->fz[fzi].count; ++j) {
            long f = o->fz[fzi].first_face + j;
            long loc = o->f_loc[f];
            for (int k = 0; k < 2; ++k) {
                long cell = k == 0 ? o->ff_c0[loc] : o->ff_c1[loc];
                long vol;
                if (cell == 0) {
                    if (bc == 31) continue;
                    long vzi = vz_find(o, o->z[zi].id);
                    vol = o->vz[vzi].first_vol + j;
                } else {
                    if (cell - 1 >= o->nfc) return fail(o, "mesh: cell index out of range");
                    long czone = o->fc_zone[cell - 1];
                    long vzi = vz_find(o, czone);
                    long zs = zone_find(o, czone);
                    vol = o->vz[vzi].first_vol + (cell - o->z[zs].first);
                }
                if (k == 0)
                    o->f_c0[f] = vol;
                else
                    o->f_c1[f] = vol;
                if (bc != 31) vol_add_face(o, vol, f);
            }
            if (face_init(o, f)) return -1;
        }
    }
    /* volume initialisation and minimum volume (:885-905) */
    double mn = -1.0;
    for (long zi = 0; zi < o->nz; ++zi) {
        long bc = o->z[zi].bc;
        if (bc == 2 || bc == 31 || bc == 32) continue;
        long vzi = vz_find(o, o->z[zi].id);
        for (long j = 0; j < o->vz[vzi].count; ++j) {
            long v = o->vz[vzi].first_vol + j;
            if (o->v_boundary[v] && o->v_fcnt[v] != 1)
                return fail(o, "mesh: boundary face zone %ld has a face without a ghost side", o->z[zi].id);
            volume_init(o, v);
            if (bc == 1 && (mn > o->V[v] || mn < 0.0)) mn = o->V[v];
        }
    }
    o->min_vol = mn;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* case setup (psstGridFV::solver_parameters and helpers)                    */
/* ------------------------------------------------------------------------ */
static int open_case_file(oracle_t *o, const char *dir, const char *name, const char *ext, strm_t *s) {
    char path[1024];
    snprintf(path, sizeof path, "%s/%s%s", dir, name, ext);
    if (load_file(path, s)) return fail(o, "Error: Could not open %s", path);
    return 0;
}

static double *U(oracle_t *o, long v) { return &o->u[v * o->dim]; }

static void prologue_w(oracle_t *o, long v) {
    int dim = o->dim;
    double vs = 0.0, rho = o->rho[v];
    double *w = &o->w[v * (dim + 2)];
    for (int j = 0; j < dim; ++j) {
        double t = U(o, v)[j];
        w[j] = rho * t;
        o->res[v * (dim + 2) + j] = 0.0;
        vs += t * t;
    }
    double E = o->cv * o->T[v] + 0.5 * vs;
    o->res[v * (dim + 2) + dim] = 0.0;
    w[dim] = rho;
    o->res[v * (dim + 2) + dim + 1] = 0.0;
    w[dim + 1] = rho * E;
}

/* ghost boundary conditions (psstBoundaryCondition.cpp) */
static void bc_dyn(oracle_t *o, vzone_t *zz, long v) {
    int dim = o->dim;
    long f = o->v_f[v][0];
    long nb = face_other(o, f, v);
    switch (zz->dyn) {
    case 23: break; /* psstSupersonicInlet::calculate_at is empty (.h:52) */
    case 26:        /* :72-80 */
        for (int j = 0; j < dim; ++j) U(o, v)[j] = U(o, nb)[j];
        o->p[v] = o->p[nb];
        break;
    case 15: { /* :108-127 */
        double vn = 0.0;
        const double *nn = &o->n[f * dim];
        for (int j = 0; j < dim; ++j) vn += U(o, nb)[j] * nn[j];
        for (int j = 0; j < dim; ++j) U(o, v)[j] = U(o, nb)[j] - vn * nn[j];
        o->p[v] = o->p[nb];
        break;
    }
    case 25: /* :212-219 */
        for (int j = 0; j < dim; ++j) U(o, v)[j] = U(o, nb)[j];
        break;
    }
}
static void bc_therm(oracle_t *o, vzone_t *zz, long v) {
    long nb = face_other(o, o->v_f[v][0], v);
    if (zz->therm == 25 || zz->therm == 18) o->T[v] = o->T[nb]; /* :285-288, :354-357 */
}

static int load_boundary(oracle_t *o, const char *dir, const char *name) {
    strm_t s;
    if (open_case_file(o, dir, name, ".bvp", &s)) return -1;
    int dim = o->dim;
    char zname[256];
    long bc;
    while (!s_eof(&s)) { /* psstFiniteVolumeGrid.cpp:418-486 */
        if (s_word(&s, zname, sizeof zname)) break;
        if (s_ulong(&s, &bc, 10)) break;
        long vzi = -1;
        for (long i = 0; i < o->nvz; ++i)
            if (!strcmp(o->z[o->vz[i].zs].name, zname)) {
                vzi = i;
                break;
            }
        if (vzi < 0) {
            free(s.buf);
            return fail(o, "Error: Could not found zone!");
        }
        vzone_t *zz = &o->vz[vzi];
        if (zz->bc == 1 || zz->bc == 2 || zz->bc == 31 || zz->bc == 32) {
            free(s.buf);
            return fail(o, "Error: Could not attach boundary condition to inner zone!");
        }
        zz->dyn = (int)bc;
        if (bc == 23) {
            o->ref_vel = 0.0;
            for (int i = 0; i < dim; ++i) {
                s_double(&s, &zz->bc_u[i]);
                o->ref_vel += zz->bc_u[i] * zz->bc_u[i];
            }
            o->ref_vel = sqrt(o->ref_vel);
            zz->bc_p = get_parameter(&s);
            for (long i = 0; i < zz->count; ++i) {
                long v = zz->first_vol + i;
                o->p[v] = zz->bc_p;
                for (int j = 0; j < dim; ++j) U(o, v)[j] = zz->bc_u[j];
            }
        } else if (bc == 26 || bc == 15) {
            for (long i = 0; i < zz->count; ++i) bc_dyn(o, zz, zz->first_vol + i);
        } else if (bc == 27) {
            free(s.buf);
            return fail(o, "Error: Wrong dimension!"); /* psstInlet ctor always throws (:147) */
        } else if (bc == 25) {
            zz->bc_p = get_parameter(&s);
            for (long i = 0; i < zz->count; ++i) {
                long v = zz->first_vol + i;
                o->p[v] = zz->bc_p;
                bc_dyn(o, zz, v);
            }
        } else {
            free(s.buf);
            return fail(o, "bvp: unsupported boundary id %ld", bc);
        }
    }
    free(s.buf);
    if (open_case_file(o, dir, name, ".btq", &s)) return -1;
    while (!s_eof(&s)) { /* :495-552 */
        if (s_word(&s, zname, sizeof zname)) break;
        if (s_ulong(&s, &bc, 10)) break;
        long vzi = -1;
        for (long i = 0; i < o->nvz; ++i)
            if (!strcmp(o->z[o->vz[i].zs].name, zname)) {
                vzi = i;
                break;
            }
        if (vzi < 0) {
            free(s.buf);
            return fail(o, "Error: Could not found zone!");
        }
        vzone_t *zz = &o->vz[vzi];
        if (zz->bc == 1 || zz->bc == 2 || zz->bc == 31 || zz->bc == 32) {
            free(s.buf);
            return fail(o, "Error: Could not attach boundary condition to inner zone!");
        }
        if (!zz->dyn) {
            free(s.buf);
            return fail(o, "btq: zone %s has no dynamic condition", zname);
        }
        zz->therm = (int)bc;
        if (bc == 11 || bc == 27) {
            double T = get_parameter(&s);
            zz->bc_T = T;
            double c = sqrt(o->gamma * o->rm * T);
            if (o->ref_vel < c) o->ref_vel = c;
            for (long i = 0; i < zz->count; ++i) o->T[zz->first_vol + i] = T;
        } else if (bc == 18 || bc == 25) {
            for (long i = 0; i < zz->count; ++i) bc_therm(o, zz, zz->first_vol + i);
        } else {
            free(s.buf);
            return fail(o, "btq: unsupported thermal id %ld", bc);
        }
        for (long i = 0; i < zz->count; ++i) {
            long v = zz->first_vol + i;
            o->rho[v] = o->p[v] / (o->rm * o->T[v]);
        }
    }
    free(s.buf);
    return 0;
}

static int load_sav(oracle_t *o, strm_t *s) {
    int dim = o->dim;
    long it = 0;
    s_ulong(s, &it, 10);
    o->iter = it;
    while (!s_eof(s)) { /* psstFiniteVolumeGrid.cpp:559-604 */
        long zid = 0, cnt = 0;
        if (s_ulong(s, &zid, 10)) break;
        if (zid == 0) break;
        long vzi = vz_find(o, zid);
        if (vzi < 0) return fail(o, "sav: unknown zone");
        s_ulong(s, &cnt, 10);
        if (cnt != o->vz[vzi].count) return fail(o, "Error! Different size of storage found!");
        for (long i = 0; i < cnt; ++i) {
            long v = o->vz[vzi].first_vol + i;
            double pp, tt;
            s_double(s, &pp);
            o->p[v] = pp;
            s_double(s, &tt);
            o->T[v] = tt;
            o->rho[v] = pp / (o->rm * tt);
            for (int j = 0; j < dim; ++j) s_double(s, &U(o, v)[j]);
        }
    }
    return 0;
}

/* psstGreenGauss::initialize (psstGradCalculation.cpp:17-72), including the
 * indexing of beta_ by the face's position inside its zone. */
static void gg_initialize(oracle_t *o) {
    int dim = o->dim;
    long maxc = 0;
    for (long i = 0; i < o->nfz; ++i)
        if (o->fz[i].count > maxc) maxc = o->fz[i].count;
    double *bz = (double *)calloc(maxc + 1, sizeof(double));
    for (long zi = 0; zi < o->nfz; ++zi) {
        if (o->fz[zi].bc == 31) continue;
        for (long i = 0; i < o->fz[zi].count; ++i) {
            long f = o->fz[zi].first_face + i;
            double d[2];
            for (int j = 0; j < 2; ++j) {
                d[j] = 0.0;
                long v = j == 0 ? o->f_c0[f] : o->f_c1[f];
                if (!o->v_boundary[v]) {
                    double dist = 0.0;
                    for (int k = 0; k < dim; ++k) {
                        double add = (o->xf[f * dim + k] - o->xc[v * dim + k]);
                        add = add * add;
                        dist += add;
                    }
                    d[j] = sqrt(dist);
                }
            }
            bz[i] = d[1] / (d[0] + d[1]);
        }
    }
    for (long zi = 0; zi < o->nfz; ++zi)
        for (long i = 0; i < o->fz[zi].count; ++i) o->beta[o->fz[zi].first_face + i] = bz[i];
    free(bz);
}

/* psstLeastSquare::initialize (:191-260); r_ indexed by zone position.
 * Coefficients per index: r11, r12, r22 and, in 3D, r13, r23, r33 and beta
 * (the Gram-Schmidt factors of the weighted normal equations, w = 1/|dx|^2;
 * Anderson & Bonhaus, Computers & Fluids 23 (1994) 1-21), computed as the
 * reference computes them for both dimensions. */
#define LSQ_NR 7
static int lsq_initialize(oracle_t *o) {
    int dim = o->dim;
    long maxc = 0;
    for (long i = 0; i < o->nvz; ++i)
        if (o->vz[i].bc == 1 && o->vz[i].count > maxc) maxc = o->vz[i].count;
    o->lsq_n = maxc;
    o->lsq_r = (double *)calloc(LSQ_NR * (maxc + 1), sizeof(double));
    for (long zi = 0; zi < o->nvz; ++zi) {
        if (o->vz[zi].bc != 1) continue;
        for (long i = 0; i < o->vz[zi].count; ++i) {
            long v = o->vz[zi].first_vol + i;
            double ca = 0.0, cb = 0.0, cd = 0.0, cc = 0.0, ce = 0.0, cg = 0.0;
            for (long j = 0; j < o->v_fcnt[v]; ++j) {
                long nb = face_other(o, o->v_f[v][j], v);
                double diff[3] = {0.0, 0.0, 0.0}, w = 0.0;
                for (int k = 0; k < dim; ++k) {
                    diff[k] = o->xc[nb * dim + k] - o->xc[v * dim + k];
                    w += diff[k] * diff[k];
                }
                double ws = 1.0 / w;
                ca += ws * diff[0] * diff[0];
                cb += ws * diff[0] * diff[1];
                cd += ws * diff[1] * diff[1];
                if (dim == 3) {
                    cc += ws * diff[0] * diff[2];
                    ce += ws * diff[1] * diff[2];
                    cg += ws * diff[2] * diff[2];
                }
            }
            double *r = &o->lsq_r[LSQ_NR * i];
            r[0] = sqrt(ca);
            r[1] = cb / r[0];
            r[2] = sqrt(cd - r[1] * r[1]);
            if (dim == 3) {
                r[3] = cc / r[0];
                r[4] = (ce - r[1] / r[0] * cc) / r[2];
                r[5] = sqrt(cg - (r[3] * r[3] + r[4] * r[4]));
                r[6] = (r[1] * r[4] - r[3] * r[2]) / (r[0] * r[2]);
            }
        }
    }
    return 0;
}

static int setup(oracle_t *o, const char *dir, const char *name) {
    int dim = o->dim;
    long nv = o->nvol;
    o->p = (double *)calloc(nv + 1, sizeof(double));
    o->T = (double *)calloc(nv + 1, sizeof(double));
    o->rho = (double *)calloc(nv + 1, sizeof(double));
    o->dt = (double *)calloc(nv + 1, sizeof(double));
    o->u = (double *)calloc((nv + 1) * dim, sizeof(double));
    o->u_old = (double *)calloc((nv + 1) * dim, sizeof(double));
    o->T_old = (double *)calloc(nv + 1, sizeof(double));
    o->w = (double *)calloc((nv + 1) * (dim + 2), sizeof(double));
    o->pw = (double *)calloc((nv + 1) * (dim + 2), sizeof(double));
    o->res = (double *)calloc((nv + 1) * (dim + 2), sizeof(double));
    o->res_conv = (double *)calloc((nv + 1) * (dim + 2), sizeof(double));
    o->g = (double *)calloc((nv + 1) * NG * dim, sizeof(double));
    o->lim = (double *)calloc((nv + 1) * NG, sizeof(double));
    o->venkat_k = 5.0;

    strm_t inp;
    if (open_case_file(o, dir, name, ".inp", &inp)) return fail(o, "Error: Could not found setting file!");
    long init_mode = (long)get_parameter(&inp);
    /* private_initialize_field (:641-717) */
    strm_t s;
    if (open_case_file(o, dir, name, ".prop", &s)) return -1;
    o->M = get_parameter(&s);
    o->cp = get_parameter(&s);
    free(s.buf);
    double R = 8.31;
    o->rm = R / o->M;
    o->gamma = o->cp / (o->cp - o->rm);
    o->cv = o->cp / o->gamma;
    if (init_mode == 0) {
        o->iter = 1;
        if (open_case_file(o, dir, name, ".par", &s)) return -1;
        double vel[3] = {0, 0, 0};
        for (int j = 0; j < dim - 1; ++j) s_double(&s, &vel[j]);
        vel[dim - 1] = get_parameter(&s);
        double Ti = get_parameter(&s);
        double pi = get_parameter(&s);
        free(s.buf);
        for (long zi = 0; zi < o->nvz; ++zi) {
            if (o->vz[zi].bc != 1) continue;
            for (long i = 0; i < o->vz[zi].count; ++i) {
                long v = o->vz[zi].first_vol + i;
                for (int j = 0; j < dim; ++j) U(o, v)[j] = vel[j];
                o->T[v] = Ti;
                o->p[v] = pi;
                o->rho[v] = pi / (o->rm * Ti);
            }
        }
    } else if (init_mode == 1) {
        if (open_case_file(o, dir, name, ".sav", &s)) return -1;
        int r = load_sav(o, &s);
        free(s.buf);
        if (r) return r;
    } else {
        return fail(o, "Error! Unknown command detected!");
    }
    if (load_boundary(o, dir, name)) return -1;

    o->CFL = get_parameter(&inp);
    o->lc = (int)(long)get_parameter(&inp);
    if (o->lc == 0 && fabs(o->ref_vel) < 1.0e-10) o->ref_vel = 1.0;
    if (o->lc < 0 || o->lc > 2) return fail(o, "inp: unknown local time mode");
    long mx = (long)get_parameter(&inp);
    o->max_iter = mx + o->iter - 1;
    o->iter_step = (long)get_parameter(&inp);
    o->rk_level = (int)(long)get_parameter(&inp);
    long rk_mode = (long)get_parameter(&inp);
    if (rk_mode == 0) {
        static const double c1[] = {1.0}, c2[] = {0.4242, 1.0}, c3[] = {0.1918, 0.4929, 1.0000},
                            c4[] = {0.1084, 0.2602, 0.5052, 1.0000},
                            c5[] = {0.0695, 0.1602, 0.2898, 0.5060, 1.0000};
        static const double *tab[] = {NULL, c1, c2, c3, c4, c5};
        if (o->rk_level < 1 || o->rk_level > 5) return fail(o, "Error: Unknow RK order!");
        for (int i = 0; i < o->rk_level; ++i) o->rk[i] = tab[o->rk_level][i];
        char *l;
        long n;
        s_getline(&inp, &l, &n);
    } else {
        if (o->rk_level < 1 || o->rk_level > 64) return fail(o, "Error! Expected Runge Kutta coefficients but empty vector found!");
        for (int i = 0; i < o->rk_level - 1; ++i) s_double(&inp, &o->rk[i]);
        o->rk[o->rk_level - 1] = get_parameter(&inp);
    }
    o->flux = (int)(long)get_parameter(&inp);
    o->order = (int)(long)get_parameter(&inp);
    o->gradm = (int)(long)get_parameter(&inp);
    o->limiter = (int)(long)get_parameter(&inp);
    free(inp.buf);
    if (o->flux < 1 || o->flux > 3) return fail(o, "Error: Unknow convective flow scheme!");
    if (o->order != 1 && o->order != 2) return fail(o, "Error! Unknown scheme order!");
    if (o->order == 2 && (o->limiter < 1 || o->limiter > 5))
        return fail(o, "second order needs a limiter 1..5 (the reference leaves it null otherwise)");
    gg_initialize(o);
    if (o->gradm != 1 && o->order == 2 && lsq_initialize(o)) return -1;
    return 0;
}

/* ------------------------------------------------------------------------ */
/* gradients                                                                 */
/* ------------------------------------------------------------------------ */
static double var_of(oracle_t *o, long v, int n) {
    int dim = o->dim;
    if (n < dim) return o->u[v * dim + n];
    if (n == dim) return o->p[v];
    if (n == dim + 1) return o->T[v];
    return o->rho[v];
}
static double *grad_of(oracle_t *o, long v, int n) { return &o->g[(v * NG + n) * o->dim]; }

/* psstGreenGauss::calculate (:80-177) */
static void gg_calculate(oracle_t *o) {
    int dim = o->dim, nvar = dim + 3;
    for (long zi = 0; zi < o->nfz; ++zi) {
        if (o->fz[zi].bc == 31) continue;
        for (long i = 0; i < o->fz[zi].count; ++i) {
            long f = o->fz[zi].first_face + i;
            long vv[2] = {o->f_c0[f], o->f_c1[f]};
            for (int j = 0; j < 2; ++j)
                for (int n = 0; n < nvar; ++n)
                    for (int k = 0; k < dim; ++k) grad_of(o, vv[j], n)[k] = 0.0;
        }
    }
    for (long zi = 0; zi < o->nfz; ++zi) {
        if (o->fz[zi].bc == 31) continue;
        for (long i = 0; i < o->fz[zi].count; ++i) {
            long f = o->fz[zi].first_face + i;
            long vv[2] = {o->f_c0[f], o->f_c1[f]};
            double gp[2];
            for (int j = 0; j < 2; ++j) gp[j] = o->S[f] / o->V[vv[j]];
            /* beta_[i] is shared across zones: the value of the last zone
             * with more than i faces (see gg_initialize) */
            double beta = o->beta[f];
            double rbeta = 1 - beta;
            for (int n = 0; n < nvar; ++n) {
                double tv = beta * var_of(o, vv[0], n) + rbeta * var_of(o, vv[1], n);
                int sign = 1;
                for (int j = 0; j < 2; ++j) {
                    sign *= -1;
                    for (int k = 0; k < dim; ++k)
                        grad_of(o, vv[j], n)[k] += sign * tv * gp[j] * o->n[f * dim + k];
                }
            }
        }
    }
}

/* psstLeastSquare::calculate (:268-368). 2D as the reference. 3D is a
 * corrected restatement: the reference leaves alpha[0..1] at zero and writes
 * alpha[3] out of bounds (:338); here alpha_1, alpha_2 are the 2D ones and
 * alpha_3 = (dz - r23/r22 dy + beta dx) / r33^2 (Anderson & Bonhaus 1994; the
 * reference's beta * dz term would not reproduce linear fields), then the
 * reference's theta corrections (:342-347). */
static void lsq_calculate(oracle_t *o) {
    int dim = o->dim, nvar = dim + 3;
    for (long zi = 0; zi < o->nvz; ++zi) {
        if (o->vz[zi].bc != 1) continue;
        for (long i = 0; i < o->vz[zi].count; ++i) {
            long v = o->vz[zi].first_vol + i;
            for (int n = 0; n < nvar; ++n)
                for (int k = 0; k < dim; ++k) grad_of(o, v, n)[k] = 0.0;
            const double *r = &o->lsq_r[LSQ_NR * i];
            for (long j = 0; j < o->v_fcnt[v]; ++j) {
                long nb = face_other(o, o->v_f[v][j], v);
                double diff[3], w = 0.0, phi[6], alpha[3], theta[3];
                for (int k = 0; k < dim; ++k) {
                    diff[k] = o->xc[nb * dim + k] - o->xc[v * dim + k];
                    w += diff[k] * diff[k];
                }
                for (int n = 0; n < nvar; ++n) phi[n] = (var_of(o, nb, n) - var_of(o, v, n));
                double ws = 1.0 / w;
                alpha[0] = diff[0] / (r[0] * r[0]);
                alpha[1] = (diff[1] - r[1] / r[0] * diff[0]) / (r[2] * r[2]);
                theta[0] = alpha[0] - r[1] / r[0] * alpha[1];
                theta[1] = alpha[1];
                if (dim == 3) {
                    alpha[2] = (diff[2] - r[4] / r[2] * diff[1] + r[6] * diff[0]) / (r[5] * r[5]);
                    theta[0] += alpha[2] * r[6];
                    theta[1] -= r[4] / r[2] * alpha[2];
                    theta[2] = alpha[2];
                }
                for (int n = 0; n < nvar; ++n)
                    for (int k = 0; k < dim; ++k) grad_of(o, v, n)[k] += ws * theta[k] * phi[n];
            }
        }
    }
}

/* Barth-Jespersen (limiter 4) / Venkatakrishnan (limiter 5) cell limiter for
 * the MUSCL extension: psi_c = min over faces of phi(Delta+, Delta-) with
 * Delta- = grad(phi)_c . (x_f - x_c). Barth & Jespersen, AIAA 89-0366;
 * Venkatakrishnan, AIAA 93-0880 (epsilon^2 = (K h)^3, h = V^(1/dim)). */
static void cell_limiters(oracle_t *o) {
    int dim = o->dim, nvar = dim + 2;
    for (long zi = 0; zi < o->nvz; ++zi) {
        if (o->vz[zi].bc != 1) continue;
        for (long i = 0; i < o->vz[zi].count; ++i) {
            long v = o->vz[zi].first_vol + i;
            double h = dim == 2 ? sqrt(o->V[v]) : cbrt(o->V[v]);
            double kh = o->venkat_k * h;
            double eps2 = kh * kh * kh;
            for (int n = 0; n < nvar; ++n) {
                double phic = var_of(o, v, n), mx = phic, mn = phic;
                for (long j = 0; j < o->v_fcnt[v]; ++j) {
                    double q = var_of(o, face_other(o, o->v_f[v][j], v), n);
                    if (q > mx) mx = q;
                    if (q < mn) mn = q;
                }
                double psi = 1.0;
                const double *g = grad_of(o, v, n);
                for (long j = 0; j < o->v_fcnt[v]; ++j) {
                    long f = o->v_f[v][j];
                    double dm = 0.0;
                    for (int k = 0; k < dim; ++k) dm += g[k] * (o->xf[f * dim + k] - o->xc[v * dim + k]);
                    double phi_f = 1.0;
                    if (dm != 0.0) {
                        double dp = dm > 0.0 ? mx - phic : mn - phic;
                        if (o->limiter == 4) {
                            double y = dp / dm;
                            phi_f = y < 1.0 ? y : 1.0;
                        } else {
                            double num = (dp * dp + eps2) + 2.0 * dm * dp;
                            double den = dp * dp + 2.0 * dm * dm + dm * dp + eps2;
                            phi_f = num / den;
                        }
                    }
                    if (phi_f < psi) psi = phi_f;
                }
                o->lim[v * NG + n] = psi;
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* reconstruction + limiters + fluxes (psstConvectiveFlow.cpp)               */
/* ------------------------------------------------------------------------ */
static double limiter_value(int type, double num, double den) { /* psstScalarLimiters.cpp:17-93 */
    double eps = 1.0e-10;
    if ((num > 0.0 && den < 0.0) || (num < 0.0 && den > 0.0)) return 0.0;
    if (fabs(den) < eps) return type == 3 ? 2.0 : 1.0;
    double r = num / den;
    if (type == 1) return (r * r + r) / (r * r + 1.0);
    if (type == 2) return r > 1.0 ? 1.0 : r;
    return 2.0 * r / (1.0 + r);
}

typedef struct {
    double p, T, rho, u[3];
} prim_t;

/* psstFirstOrderReconstructor / psstReconstructorDM::reconstruct_vals
 * (psstValueReconstructor.cpp:28-48, 70-134); MUSCL for limiters 4/5. */
static void reconstruct(oracle_t *o, long f, prim_t r[2]) {
    int dim = o->dim;
    long vv[2] = {o->f_c0[f], o->f_c1[f]};
    for (int j = 0; j < 2; ++j) {
        r[j].p = o->p[vv[j]];
        r[j].T = o->T[vv[j]];
        r[j].rho = o->rho[vv[j]];
        for (int i = 0; i < dim; ++i) r[j].u[i] = U(o, vv[j])[i];
    }
    if (o->order == 1) return;
    double *pv[2][5];
    for (int j = 0; j < 2; ++j) {
        for (int i = 0; i < dim; ++i) pv[j][i] = &r[j].u[i];
        pv[j][dim] = &r[j].p;
        pv[j][dim + 1] = &r[j].T;
    }
    if (o->limiter >= 4) { /* phi_f = phi_c + (psi grad phi) . (x_f - x_c) */
        for (int j = 0; j < 2; ++j)
            for (int i = 0; i < dim + 2; ++i) {
                const double *g = grad_of(o, vv[j], i);
                const double psi = o->lim[vv[j] * NG + i];
                double d = 0.0;
                for (int k = 0; k < dim; ++k) d += (g[k] * psi) * (o->xf[f * dim + k] - o->xc[vv[j] * dim + k]);
                *pv[j][i] += d;
            }
    } else {
        double R[3];
        for (int j = 0; j < dim; ++j) R[j] = o->xc[vv[0] * dim + j] - o->xc[vv[1] * dim + j];
        for (int i = 0; i < dim + 2; ++i) {
            double dl = 0.0, dr = 0.0;
            const double *g1 = grad_of(o, vv[1], i), *g0 = grad_of(o, vv[0], i);
            for (int k = 0; k < dim; ++k) {
                dl += g1[k] * R[k];
                dr += g0[k] * R[k];
            }
            double v0 = *pv[0][i], v1 = *pv[1][i];
            double vlm = v1 - (2.0 * dl - (v0 - v1));
            double vlp = v0;
            double vrm = v1;
            double vrp = v0 + (2.0 * dr - (v0 - v1));
            double nl = vlp - v1, dnl = v1 - vlm;
            double nr = vrm - v0, dnr = v0 - vrp;
            *pv[0][i] += 0.5 * limiter_value(o->limiter, nr, dnr) * dnr;
            *pv[1][i] += 0.5 * limiter_value(o->limiter, nl, dnl) * dnl;
        }
    }
    for (int j = 0; j < 2; ++j) r[j].rho = r[j].p / (o->rm * r[j].T);
}

static double roe_avg(double lv, double rv, double ld, double rd) { /* :13-24 */
    double l = sqrt(ld), r = sqrt(rd);
    double num = lv * l + rv * r;
    double den = (l + r);
    return num / den;
}

static int face_flux(oracle_t *o, long f, double *flow) {
    int dim = o->dim, ws = dim + 2;
    const double *nn = &o->n[f * dim];
    double cp = o->cp, cv = o->cv, rm = o->rm, gamma = o->gamma;
    prim_t r[2];
    reconstruct(o, f, r);
    double vn[2], vel[2][3], a[2], H[2], E[2], fi[2][MAXV], wi[2][MAXV], M[2];
    for (int j = 0; j < 2; ++j) {
        vn[j] = 0.0;
        double vs = 0.0;
        for (int k = 0; k < dim; ++k) {
            vel[j][k] = r[j].u[k];
            vn[j] += vel[j][k] * nn[k];
            vs += vel[j][k] * vel[j][k];
        }
        a[j] = sqrt(gamma * rm * r[j].T);
        H[j] = cp * r[j].T + 0.5 * vs;
        if (o->flux == 1) {
            M[j] = vn[j] / a[j];
            continue;
        }
        E[j] = cv * r[j].T + 0.5 * vs;
        for (int k = 0; k < dim; ++k) {
            fi[j][k] = r[j].rho * vel[j][k] * vn[j] + r[j].p * nn[k];
            wi[j][k] = r[j].rho * vel[j][k];
        }
        wi[j][dim] = r[j].rho;
        wi[j][dim + 1] = r[j].rho * E[j];
        fi[j][dim] = r[j].rho * vn[j];
        fi[j][dim + 1] = r[j].rho * vn[j] * H[j];
    }
    if (o->flux == 1) { /* psstConvectiveAUSM::calculate :804-851 */
        double Ms[2], ps[2];
        if (M[1] >= 1.0) {
            Ms[1] = M[1];
            ps[1] = r[1].p;
        } else if (M[1] <= -1.0) {
            Ms[1] = 0.0;
            ps[1] = 0.0;
        } else {
            Ms[1] = 0.25 * (M[1] + 1.0) * (M[1] + 1.0);
            ps[1] = 0.25 * r[1].p * (M[1] + 1.0) * (M[1] + 1.0) * (2.0 - M[1]);
        }
        if (M[0] >= 1.0) {
            Ms[0] = 0.0;
            ps[0] = 0.0;
        } else if (M[0] <= -1.0) {
            Ms[0] = M[0];
            ps[0] = r[0].p;
        } else {
            Ms[0] = -0.25 * (M[0] - 1.0) * (M[0] - 1.0);
            ps[0] = 0.25 * r[0].p * (M[0] - 1.0) * (M[0] - 1.0) * (2.0 + M[0]);
        }
        double Mf = Ms[0] + Ms[1], pf = ps[0] + ps[1];
        int sd = Mf > 0.0 ? 1 : 0;
        double t = Mf * a[sd] * r[sd].rho;
        for (int j = 0; j < dim; ++j) {
            double pfl = pf * nn[j];
            flow[j] = t * vel[sd][j] + pfl;
        }
        flow[dim] = t;
        flow[dim + 1] = t * H[sd];
        return 0;
    }
    double HR = roe_avg(H[1], H[0], r[1].rho, r[0].rho);
    double vRn = 0.0, vs = 0.0, vR[3];
    for (int k = 0; k < dim; ++k) {
        vR[k] = roe_avg(vel[1][k], vel[0][k], r[1].rho, r[0].rho);
        vRn += vR[k] * nn[k];
        vs += vR[k] * vR[k];
    }
    double aR = sqrt((gamma - 1.0) * (HR - 0.5 * vs));
    double s[2], t;
    s[1] = vn[1] - a[1];
    t = vRn - aR;
    if (s[1] > t) s[1] = t;
    s[0] = vn[0] + a[0];
    t = vRn + aR;
    if (s[0] < t) s[0] = t;
    if (o->flux == 2) { /* HLL :268-286 */
        if (s[1] >= 0.0) {
            for (int j = 0; j < ws; ++j) flow[j] = fi[1][j];
        } else if (s[1] <= 0.0 && s[0] >= 0.0) {
            for (int j = 0; j < ws; ++j)
                flow[j] = (s[0] * fi[1][j] - s[1] * fi[0][j] + s[0] * s[1] * (wi[0][j] - wi[1][j])) / (s[0] - s[1]);
        } else if (s[0] <= 0.0) {
            for (int j = 0; j < ws; ++j) flow[j] = fi[0][j];
        } else {
            return fail(o, "Error: Could not calculate convective HLL flow!");
        }
        return 0;
    }
    /* HLLC :552-585 */
    double p0 = r[0].p, p1 = r[1].p, d0 = r[0].rho, d1 = r[1].rho;
    double sh = (p0 - p1 + d1 * vn[1] * (s[1] - vn[1]) - d0 * vn[0] * (s[0] - vn[0])) /
                (d1 * (s[1] - vn[1]) - d0 * (s[0] - vn[0]));
    if (s[1] >= 0.0) {
        for (int j = 0; j < ws; ++j) flow[j] = fi[1][j];
    } else if ((s[1] <= 0.0 && sh >= 0.0) || (sh <= 0.0 && s[0] >= 0.0)) {
        int sd = (s[1] <= 0.0 && sh >= 0.0) ? 1 : 0;
        double tt = s[sd] - sh;
        double pr = r[sd].p, dd = r[sd].rho;
        for (int j = 0; j < dim; ++j)
            flow[j] = (sh * (s[sd] * wi[sd][j] - fi[sd][j]) +
                       s[sd] * (pr + dd * (s[sd] - vn[sd]) * (sh - vn[sd])) * nn[j]) / tt;
        flow[dim] = (sh * (s[sd] * wi[sd][dim] - fi[sd][dim])) / tt;
        flow[dim + 1] = (sh * (s[sd] * wi[sd][dim + 1] - fi[sd][dim + 1]) +
                         s[sd] * (pr + dd * (s[sd] - vn[sd]) * (sh - vn[sd])) * sh) / tt;
    } else if (s[0] <= 0.0) {
        for (int j = 0; j < ws; ++j) flow[j] = fi[0][j];
    } else {
        return fail(o, "Error: Could not calculate convective HLLC flow!");
    }
    return 0;
}

/* boundary faces: physical flux of the ghost state (:123-202) */
static void boundary_flux(oracle_t *o, long f, long g, double *flow) {
    int dim = o->dim;
    const double *nn = &o->n[f * dim];
    double vn = 0.0, vs = 0.0, vel[3];
    double p = o->p[g], rho = o->rho[g], T = o->T[g];
    for (int k = 0; k < dim; ++k) {
        vel[k] = U(o, g)[k];
        vn += vel[k] * nn[k];
        vs += vel[k] * vel[k];
    }
    double H = o->cp * T + 0.5 * vs;
    for (int k = 0; k < dim; ++k) flow[k] = rho * vel[k] * vn + p * nn[k];
    flow[dim] = rho * vn;
    flow[dim + 1] = rho * vn * H;
}

static int convective(oracle_t *o) {
    int dim = o->dim, ws = dim + 2;
    double flow[MAXV];
    for (long zi = 0; zi < o->nfz; ++zi) {
        long bc = o->fz[zi].bc;
        if (bc == 31) continue;
        for (long i = 0; i < o->fz[zi].count; ++i) {
            long f = o->fz[zi].first_face + i;
            double S = o->S[f];
            long v0 = o->f_c0[f], v1 = o->f_c1[f];
            if (bc != 2) {
                if (o->v_boundary[v0]) {
                    boundary_flux(o, f, v0, flow);
                    for (int k = 0; k < ws; ++k) o->res[v1 * ws + k] += flow[k] * S;
                } else {
                    boundary_flux(o, f, v1, flow);
                    for (int k = 0; k < ws; ++k) o->res[v0 * ws + k] -= flow[k] * S;
                }
            } else {
                if (face_flux(o, f, flow)) return -1;
                int sign = 1;
                long vv[2] = {v0, v1};
                for (int j = 0; j < 2; ++j) {
                    sign = (-1) * sign;
                    for (int k = 0; k < ws; ++k) o->res[vv[j] * ws + k] += sign * flow[k] * S;
                }
            }
        }
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* local time step (psstLocalTimeCalculation.cpp)                            */
/* ------------------------------------------------------------------------ */
static void local_time(oracle_t *o, long v, const double *uu, const double *TT) {
    int dim = o->dim;
    double vol = o->V[v];
    if (o->lc == 1) { /* psstLocalAccTime1::calculate_at :90-131 */
        double nn_nb = 0.0, den = 0.0;
        double c = sqrt(o->gamma * o->rm * TT[v]);
        for (long j = 0; j < o->v_fcnt[v]; ++j) {
            double nvel = 0.0;
            long f = o->v_f[v][j];
            long nb = face_other(o, f, v);
            double cn = (sqrt(o->gamma * o->rm * TT[nb]) + c) * 0.5;
            for (int k = 0; k < dim; ++k) {
                double t = o->n[f * dim + k];
                nvel += uu[v * dim + k] * t;
                nn_nb += uu[nb * dim + k] * t;
            }
            nn_nb = (nn_nb + nvel) * 0.5;
            den += (fabs(nn_nb) + cn) * o->S[f];
        }
        o->dt[v] = o->CFL * vol / den;
    } else if (o->lc == 2) { /* psstLocalAccTime2::calculate_at :175-213 */
        double s[3] = {0, 0, 0}, den = 0.0;
        double c = sqrt(o->gamma * o->rm * TT[v]);
        for (long j = 0; j < o->v_fcnt[v]; ++j) {
            long f = o->v_f[v][j];
            for (int k = 0; k < dim; ++k) s[k] += o->S[f] * fabs(o->n[f * dim + k]);
        }
        for (int j = 0; j < dim; ++j) den += (fabs(uu[v * dim + j]) + c) * s[j] * 0.5;
        o->dt[v] = o->CFL * vol / den;
    }
}

static void uniform_time(oracle_t *o) { /* psstUniformTime::initialize :21-43 */
    double dtv;
    if (o->dim == 2)
        dtv = o->CFL * sqrt(o->min_vol) / o->ref_vel;
    else
        dtv = o->CFL * pow(o->min_vol, 1.0 / 3.0) / o->ref_vel;
    for (long zi = 0; zi < o->nvz; ++zi)
        if (o->vz[zi].bc == 1)
            for (long i = 0; i < o->vz[zi].count; ++i) o->dt[o->vz[zi].first_vol + i] = dtv;
}

/* ------------------------------------------------------------------------ */
/* the explicit_solve loop (psstFiniteVolumeGrid.cpp:248-401)                */
/* ------------------------------------------------------------------------ */
int oracle_run(oracle_t *o, int n_iter, double *res_linf, double *res_l2) {
    int dim = o->dim, ws = dim + 2;
    long nint = 0;
    for (long zi = 0; zi < o->nvz; ++zi)
        if (o->vz[zi].bc == 1) nint += o->vz[zi].count;
    for (int it = 0; it < n_iter; ++it) {
        double rmax[MAXV] = {0, 0, 0, 0, 0}, l2max[MAXV] = {0, 0, 0, 0, 0};
        if (o->order == 2) {
            if (o->gradm == 1)
                gg_calculate(o);
            else
                lsq_calculate(o);
            if (o->limiter >= 4) cell_limiters(o);
        }
        for (int k = 0; k < o->rk_level; ++k) {
            if (convective(o)) return -1;
            if (o->lc == 1 && o->lc1_jacobi) {
                memcpy(o->u_old, o->u, sizeof(double) * o->nvol * dim);
                memcpy(o->T_old, o->T, sizeof(double) * o->nvol);
            }
            double l2[MAXV] = {0, 0, 0, 0, 0};
            for (long zi = 0; zi < o->nvz; ++zi) {
                if (o->vz[zi].bc != 1) continue;
                for (long i = 0; i < o->vz[zi].count; ++i) {
                    long v = o->vz[zi].first_vol + i;
                    double vol = o->V[v];
                    if (o->lc == 1 && o->lc1_jacobi)
                        local_time(o, v, o->u_old, o->T_old);
                    else
                        local_time(o, v, o->u, o->T);
                    double *w = &o->w[v * ws], *pw = &o->pw[v * ws], *rs = &o->res[v * ws];
                    for (int j = 0; j < ws; ++j) {
                        if (k == 0) pw[j] = w[j];
                        w[j] = pw[j] - o->dt[v] * o->rk[k] * rs[j] / vol;
                        if (rmax[j] < fabs(rs[j])) rmax[j] = fabs(rs[j]);
                        l2[j] += rs[j] * rs[j];
                        rs[j] = 0.0;
                    }
                    double rho = w[dim];
                    o->rho[v] = rho;
                    double vs = 0.0;
                    for (int j = 0; j < dim; ++j) {
                        U(o, v)[j] = w[j] / rho;
                        double vel = U(o, v)[j];
                        vs += vel * vel;
                    }
                    o->T[v] = ((w[dim + 1] / rho) - (vs * 0.5)) / o->cv;
                    o->p[v] = rho * o->rm * o->T[v];
                }
            }
            for (int j = 0; j < ws; ++j) {
                double r = sqrt(l2[j] / (double)(nint ? nint : 1));
                if (r > l2max[j]) l2max[j] = r;
            }
            for (long zi = 0; zi < o->nvz; ++zi) { /* :351-366 */
                if (o->vz[zi].bc == 1 || o->vz[zi].bc == 32) continue;
                for (long i = 0; i < o->vz[zi].count; ++i) {
                    long v = o->vz[zi].first_vol + i;
                    bc_dyn(o, &o->vz[zi], v);
                    bc_therm(o, &o->vz[zi], v);
                    o->rho[v] = o->p[v] / (o->T[v] * o->rm);
                }
            }
        }
        if (res_linf)
            for (int j = 0; j < ws; ++j) res_linf[(long)it * ws + j] = rmax[j];
        if (res_l2)
            for (int j = 0; j < ws; ++j) res_l2[(long)it * ws + j] = l2max[j];
        o->iter++;
    }
    return 0;
}

/* One stage's convective residual of the current state, as the reference
 * holds it between its face loop (psstConvectiveFlow.cpp:289-299, after the
 * iteration's gradients, psstFiniteVolumeGrid.cpp:307-311) and the update
 * loop that consumes and zeroes it (:324-333): copied to res_conv
 * ("vol_res"); the state and the running residual are left untouched. */
int oracle_convective(oracle_t *o) {
    long n = (o->nvol + 1) * (o->dim + 2);
    if (o->order == 2) {
        if (o->gradm == 1)
            gg_calculate(o);
        else
            lsq_calculate(o);
        if (o->limiter >= 4) cell_limiters(o);
    }
    memset(o->res, 0, sizeof(double) * n);
    if (convective(o)) return -1;
    memcpy(o->res_conv, o->res, sizeof(double) * n);
    memset(o->res, 0, sizeof(double) * n);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* API                                                                       */
/* ------------------------------------------------------------------------ */
oracle_t *oracle_open(const char *mesh_path, const char *case_dir, const char *case_name, char *err,
                      int errlen) {
    oracle_t *o = (oracle_t *)calloc(1, sizeof(oracle_t));
    if (read_mesh(o, mesh_path) || build_fv(o) || setup(o, case_dir, case_name)) {
        if (err) snprintf(err, errlen, "%s", o->err);
        oracle_close(o);
        return NULL;
    }
    if (o->lc == 0) uniform_time(o);
    for (long v = 0; v < o->nvol; ++v) prologue_w(o, v);
    return o;
}

int oracle_set(oracle_t *o, const char *key, double value) {
    if (!strcmp(key, "lc1_jacobi"))
        o->lc1_jacobi = value != 0.0;
    else if (!strcmp(key, "limiter")) {
        o->limiter = (int)value;
        if (o->order == 2 && o->gradm != 1 && !o->lsq_r && lsq_initialize(o)) return -1;
    } else if (!strcmp(key, "venkat_k"))
        o->venkat_k = value;
    else if (!strcmp(key, "order"))
        o->order = (int)value;
    else
        return fail(o, "unknown option %s", key);
    return 0;
}

const char *oracle_error(const oracle_t *o) { return o->err; }
int oracle_dim(const oracle_t *o) { return o->dim; }
int oracle_nvol(const oracle_t *o) { return (int)o->nvol; }
int oracle_nface(const oracle_t *o) { return (int)o->nface; }
int oracle_iter(const oracle_t *o) { return (int)o->iter; }

long oracle_get(const oracle_t *o, const char *name, double *out, long cap) {
    int dim = o->dim;
    long nv = o->nvol, nf = o->nface, cnt = 0;
#define COPY(N, EXPR)                             \
    do {                                          \
        cnt = (N);                                \
        if (out && cap >= cnt)                    \
            for (long i = 0; i < cnt; ++i) out[i] = (EXPR); \
        return cnt;                               \
    } while (0)
    if (!strcmp(name, "vol_p")) COPY(nv, o->p[i]);
    if (!strcmp(name, "vol_T")) COPY(nv, o->T[i]);
    if (!strcmp(name, "vol_rho")) COPY(nv, o->rho[i]);
    if (!strcmp(name, "vol_u")) COPY(nv * dim, o->u[i]);
    if (!strcmp(name, "vol_w")) COPY(nv * (dim + 2), o->w[i]);
    if (!strcmp(name, "vol_prev_w")) COPY(nv * (dim + 2), o->pw[i]);
    if (!strcmp(name, "vol_dt")) COPY(nv, o->dt[i]);
    if (!strcmp(name, "vol_res")) COPY(nv * (dim + 2), o->res_conv[i]);
    if (!strcmp(name, "vol_V")) COPY(nv, o->V[i]);
    if (!strcmp(name, "vol_x")) COPY(nv * dim, o->xc[i]);
    if (!strcmp(name, "vol_grad_u")) COPY(nv * dim * dim, o->g[((i / (dim * dim)) * NG + (i % (dim * dim)) / dim) * dim + i % dim]);
    if (!strcmp(name, "vol_grad_p")) COPY(nv * dim, o->g[((i / dim) * NG + dim) * dim + i % dim]);
    if (!strcmp(name, "vol_grad_T")) COPY(nv * dim, o->g[((i / dim) * NG + dim + 1) * dim + i % dim]);
    if (!strcmp(name, "vol_grad_rho")) COPY(nv * dim, o->g[((i / dim) * NG + dim + 2) * dim + i % dim]);
    if (!strcmp(name, "vol_lim")) COPY(nv * (dim + 2), o->lim[(i / (dim + 2)) * NG + i % (dim + 2)]);
    /* gradients as the reconstruction uses them: times psi with limiters 4/5 */
    if (!strcmp(name, "vol_lgrad_u"))
        COPY(nv * dim * dim, o->g[((i / (dim * dim)) * NG + (i % (dim * dim)) / dim) * dim + i % dim] *
                                 (o->limiter >= 4 ? o->lim[(i / (dim * dim)) * NG + (i % (dim * dim)) / dim] : 1.0));
    if (!strcmp(name, "vol_lgrad_p"))
        COPY(nv * dim, o->g[((i / dim) * NG + dim) * dim + i % dim] * (o->limiter >= 4 ? o->lim[(i / dim) * NG + dim] : 1.0));
    if (!strcmp(name, "vol_lgrad_T"))
        COPY(nv * dim, o->g[((i / dim) * NG + dim + 1) * dim + i % dim] *
                           (o->limiter >= 4 ? o->lim[(i / dim) * NG + dim + 1] : 1.0));
    if (!strcmp(name, "vol_zone")) COPY(nv, (double)o->vz[o->v_vz[i]].id);
    if (!strcmp(name, "vol_bc")) COPY(nv, (double)o->vz[o->v_vz[i]].bc);
    if (!strcmp(name, "vol_boundary")) COPY(nv, (double)o->v_boundary[i]);
    if (!strcmp(name, "vol_nfaces")) COPY(nv, (double)o->v_fcnt[i]);
    if (!strcmp(name, "face_S")) COPY(nf, o->S[i]);
    if (!strcmp(name, "face_n")) COPY(nf * dim, o->n[i]);
    if (!strcmp(name, "face_x")) COPY(nf * dim, o->xf[i]);
    if (!strcmp(name, "face_beta")) COPY(nf, o->beta[i]);
    if (!strcmp(name, "face_zone")) COPY(nf, (double)o->fz[o->f_fz[i]].id);
    if (!strcmp(name, "face_bc")) COPY(nf, (double)o->fz[o->f_fz[i]].bc);
    if (!strcmp(name, "face_c0")) COPY(nf, (double)o->f_c0[i]);
    if (!strcmp(name, "face_c1")) COPY(nf, (double)o->f_c1[i]);
    if (!strcmp(name, "gas")) {
        double g4[4] = {o->rm, o->cp, o->cv, o->gamma};
        COPY(4, g4[i]);
    }
    if (!strcmp(name, "min_vol")) COPY(1, o->min_vol);
    if (!strcmp(name, "rk")) COPY(o->rk_level, o->rk[i]);
    if (!strcmp(name, "scheme")) {
        double sc[10] = {o->CFL, o->lc, o->rk_level, o->flux, o->order, o->gradm, o->limiter, o->ref_vel,
                         (double)o->iter, (double)o->max_iter};
        COPY(10, sc[i]);
    }
#undef COPY
    return -1;
}

int oracle_set_prim(oracle_t *o, const double *p, const double *T, const double *u) {
    int dim = o->dim;
    for (long v = 0; v < o->nvol; ++v) {
        o->p[v] = p[v];
        o->T[v] = T[v];
        o->rho[v] = p[v] / (o->rm * T[v]);
        for (int j = 0; j < dim; ++j) o->u[v * dim + j] = u[v * dim + j];
        prologue_w(o, v);
    }
    return 0;
}

int oracle_write_sav(const oracle_t *o, const char *path) {
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    int dim = o->dim;
    fprintf(f, "%ld\n", o->iter);
    for (long zi = 0; zi < o->nvz; ++zi) {
        if (o->vz[zi].bc != 1) continue;
        fprintf(f, "%ld\n%ld\n", o->vz[zi].id, o->vz[zi].count);
        for (long i = 0; i < o->vz[zi].count; ++i) {
            long v = o->vz[zi].first_vol + i;
            fprintf(f, "%.11f %.11f ", o->p[v], o->T[v]);
            for (int j = 0; j < dim; ++j) fprintf(f, "%.11f ", o->u[v * dim + j]);
            fprintf(f, "\n");
        }
    }
    fprintf(f, "0");
    fclose(f);
    return 0;
}

void oracle_close(oracle_t *o) {
    if (!o) return;
    free(o->vx);
    free(o->ff_ptr);
    free(o->ff_nodes);
    free(o->ff_c0);
    free(o->ff_c1);
    free(o->ff_zone);
    free(o->fc_zone);
    free(o->z);
    free(o->vz);
    free(o->fz);
    if (o->v_f)
        for (long v = 0; v < o->nvol; ++v) free(o->v_f[v]);
    free(o->v_f);
    free(o->v_fcnt);
    free(o->v_fcap);
    free(o->v_boundary);
    free(o->v_vz);
    free(o->V);
    free(o->xc);
    free(o->f_c0);
    free(o->f_c1);
    free(o->f_fz);
    free(o->f_loc);
    free(o->S);
    free(o->n);
    free(o->xf);
    free(o->beta);
    free(o->p);
    free(o->T);
    free(o->rho);
    free(o->u);
    free(o->u_old);
    free(o->T_old);
    free(o->w);
    free(o->pw);
    free(o->res);
    free(o->res_conv);
    free(o->dt);
    free(o->g);
    free(o->lim);
    free(o->lsq_r);
    free(o);
}

#ifdef PSST_ORACLE_MAIN
/* CLI mirroring main.cpp: reads ./problem_manager (mesh, case), runs max_iter
 * iterations, writes <case>.sav and <case>_residual.dat (residual columns as
 * the reference prints them; the wall-time column is the oracle's own). */
#include <time.h>
int main(int argc, char **argv) {
    const char *pm = argc > 1 ? argv[1] : "problem_manager";
    FILE *f = fopen(pm, "r");
    if (!f) {
        fprintf(stderr, "Error: Could not open problem_manager file!");
        return 1;
    }
    char mesh[512], cs[512];
    if (fscanf(f, "%511s %511s", mesh, cs) != 2) {
        fclose(f);
        return 1;
    }
    fclose(f);
    char err[512];
    oracle_t *o = oracle_open(mesh, ".", cs, err, sizeof err);
    if (!o) {
        fprintf(stderr, "%s\n", err);
        return 1;
    }
    int ws = o->dim + 2;
    long n = o->max_iter - o->iter + 1;
    char path[600];
    snprintf(path, sizeof path, "%s_residual.dat", cs);
    FILE *rf = fopen(path, "w");
    struct timespec t0, t1;
    clock_gettime(CLOCK_MONOTONIC, &t0);
    for (long i = 0; i < n; ++i) {
        double r[MAXV];
        long it = o->iter;
        if (oracle_run(o, 1, r, NULL)) {
            fprintf(stderr, "%s\n", o->err);
            return 1;
        }
        clock_gettime(CLOCK_MONOTONIC, &t1);
        long ms = (t1.tv_sec - t0.tv_sec) * 1000 + (t1.tv_nsec - t0.tv_nsec) / 1000000;
        fprintf(rf, "%ld %.11e ", it, ms / 1000.0);
        for (int j = 0; j < ws; ++j) fprintf(rf, " %.3e", r[j]);
        fprintf(rf, "\n");
    }
    fclose(rf);
    snprintf(path, sizeof path, "%s.sav", cs);
    oracle_write_sav(o, path);
    oracle_close(o);
    return 0;
}
#endif
