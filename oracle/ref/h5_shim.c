/*
 * In-memory HDF5 stand-in (hdf5.h) and entry points that run the reference's
 * data readers and view generator on arrays given by the caller.  Test
 * infrastructure only.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "hdf5.h"

#define MAXD 8
#define MAXS 32

static struct {
    char file[64], name[64];
    const void *data;
    int bytes, rank;
    hsize_t dims[3];
} g_dsets[MAXD];
static int g_ndsets;

/* spaces: dims plus the selected hyperslab */
static struct {
    int used, rank;
    hsize_t dims[3], start[3], count[3];
} g_spaces[MAXS];

static const char *g_files[MAXD];
static int g_nfiles;

int ref_h5_register(const char *file, const char *dset, const void *data, int elem_bytes, int rank,
                    const hsize_t *dims)
{
    if (g_ndsets >= MAXD || rank < 1 || rank > 3) return -1;
    strncpy(g_dsets[g_ndsets].file, file, 63);
    strncpy(g_dsets[g_ndsets].name, dset, 63);
    g_dsets[g_ndsets].data = data;
    g_dsets[g_ndsets].bytes = elem_bytes;
    g_dsets[g_ndsets].rank = rank;
    for (int i = 0; i < rank; i++) g_dsets[g_ndsets].dims[i] = dims[i];
    g_ndsets++;
    return 0;
}

void ref_h5_clear(void)
{
    g_ndsets = 0;
    g_nfiles = 0;
    memset(g_spaces, 0, sizeof g_spaces);
}

hid_t H5Fopen(const char *name, unsigned flags, hid_t plist)
{
    (void)flags;
    (void)plist;
    if (g_nfiles >= MAXD) return -1;
    g_files[g_nfiles] = name;
    return g_nfiles++;
}

hid_t H5Dopen(hid_t file, const char *name, hid_t plist)
{
    (void)plist;
    if (file < 0 || file >= g_nfiles) return -1;
    for (int i = 0; i < g_ndsets; i++)
        if (!strcmp(g_dsets[i].file, g_files[file]) && !strcmp(g_dsets[i].name, name)) return i;
    fprintf(stderr, "h5 stand-in: no dataset %s in %s\n", name, g_files[file]);
    return -1;
}

static hid_t new_space(int rank, const hsize_t *dims)
{
    for (int s = 0; s < MAXS; s++)
        if (!g_spaces[s].used) {
            g_spaces[s].used = 1;
            g_spaces[s].rank = rank;
            for (int i = 0; i < rank; i++) {
                g_spaces[s].dims[i] = dims[i];
                g_spaces[s].start[i] = 0;
                g_spaces[s].count[i] = dims[i];
            }
            return s;
        }
    return -1;
}

hid_t H5Dget_space(hid_t dset)
{
    if (dset < 0 || dset >= g_ndsets) return -1;
    return new_space(g_dsets[dset].rank, g_dsets[dset].dims);
}

int H5Sget_simple_extent_ndims(hid_t space) { return space < 0 ? -1 : g_spaces[space].rank; }

int H5Sget_simple_extent_dims(hid_t space, hsize_t *dims, hsize_t *maxdims)
{
    (void)maxdims;
    if (space < 0) return -1;
    for (int i = 0; i < g_spaces[space].rank; i++) dims[i] = g_spaces[space].dims[i];
    return g_spaces[space].rank;
}

herr_t H5Sselect_hyperslab(hid_t space, H5S_seloper_t op, const hsize_t *start, const hsize_t *stride,
                           const hsize_t *count, const hsize_t *block)
{
    (void)op;
    if (space < 0 || stride || block) return -1;
    for (int i = 0; i < g_spaces[space].rank; i++) {
        if (start[i] + count[i] > g_spaces[space].dims[i]) return -1;
        g_spaces[space].start[i] = start[i];
        g_spaces[space].count[i] = count[i];
    }
    return 0;
}

hid_t H5Screate_simple(int rank, const hsize_t *dims, const hsize_t *maxdims)
{
    (void)maxdims;
    return new_space(rank, dims);
}

herr_t H5Dread(hid_t dset, hid_t mem_type, hid_t mem_space, hid_t file_space, hid_t plist, void *buf)
{
    (void)mem_space;
    (void)plist;
    if (dset < 0 || file_space < 0 || mem_type != g_dsets[dset].bytes) return -1;
    const int b = g_dsets[dset].bytes;
    const hsize_t *d = g_dsets[dset].dims, *st = g_spaces[file_space].start, *c = g_spaces[file_space].count;
    const char *src = (const char *)g_dsets[dset].data;
    char *dst = (char *)buf;
    /* rank 3 (the readers' datasets); lower ranks are padded with leading 1s */
    hsize_t D[3] = {1, 1, 1}, S[3] = {0, 0, 0}, C[3] = {1, 1, 1};
    const int r = g_dsets[dset].rank;
    for (int i = 0; i < r; i++) {
        D[3 - r + i] = d[i];
        S[3 - r + i] = st[i];
        C[3 - r + i] = c[i];
    }
    for (hsize_t i = 0; i < C[0]; i++)
        for (hsize_t j = 0; j < C[1]; j++) {
            const size_t off = (((S[0] + i) * D[1] + S[1] + j) * D[2] + S[2]) * (size_t)b;
            memcpy(dst, src + off, C[2] * (size_t)b);
            dst += C[2] * (size_t)b;
        }
    return 0;
}

herr_t H5Sclose(hid_t space)
{
    if (space >= 0) g_spaces[space].used = 0;
    return 0;
}
herr_t H5Dclose(hid_t dset)
{
    (void)dset;
    return 0;
}
herr_t H5Fclose(hid_t file)
{
    (void)file;
    return 0;
}

/* ---- the reference's functions, on caller arrays ---- */
int32_t read_data(char data_filename[], char whites_filename[], char darks_filename[], float *projections,
                  float *weights, int32_t datafile_row0, int32_t proj_rows, int32_t proj_cols, int32_t proj_start,
                  int32_t proj_num, FILE *debug_file_ptr);
int32_t read_ProjWeightData(char data_filename[], float *projections, float *weights, int32_t datafile_row0,
                            int32_t proj_rows, int32_t proj_cols, int32_t proj_start, int32_t proj_num,
                            FILE *debug_file_ptr);
int32_t gen_interlaced_views_0_to_Inf(float *views, float *times, int32_t K, int32_t N_theta, int32_t proj_start,
                                      int32_t N_p, float min_acq_time, float rot_speed, FILE *debug_file_ptr);

static FILE *sink(void)
{
    static FILE *f;
    if (!f) f = fopen("/dev/null", "w");
    return f;
}

/* APS reader (aps_data/XT_HDFIO.c read_data): counts [n][rows][cols], whites
 * [nw][rows][cols], darks [nd][rows][cols], uint16 */
int ref_read_aps(const uint16_t *counts, int n, const uint16_t *whites, int nw, const uint16_t *darks, int nd,
                 int rows, int cols, int datafile_row0, int proj_rows, int proj_cols, int proj_start, int proj_num,
                 float *projections, float *weights)
{
    ref_h5_clear();
    hsize_t dc[3] = {(hsize_t)n, (hsize_t)rows, (hsize_t)cols}, dw[3] = {(hsize_t)nw, (hsize_t)rows, (hsize_t)cols},
            dd[3] = {(hsize_t)nd, (hsize_t)rows, (hsize_t)cols};
    ref_h5_register("data", "/exchange/data", counts, 2, 3, dc);
    ref_h5_register("white", "/exchange/data_white", whites, 2, 3, dw);
    ref_h5_register("dark", "/exchange/data_dark", darks, 2, 3, dd);
    char a[] = "data", b[] = "white", c[] = "dark";
    return read_data(a, b, c, projections, weights, datafile_row0, proj_rows, proj_cols, proj_start, proj_num,
                     sink());
}

/* standard reader (std_data/XT_HDFIO.c read_ProjWeightData): float
 * projections and weights [n][rows][cols] */
int ref_read_std(const float *projs, const float *wts, int n, int rows, int cols, int datafile_row0, int proj_rows,
                 int proj_cols, int proj_start, int proj_num, float *projections, float *weights)
{
    ref_h5_clear();
    hsize_t d[3] = {(hsize_t)n, (hsize_t)rows, (hsize_t)cols};
    ref_h5_register("data", "/projections", projs, 4, 3, d);
    ref_h5_register("data", "/weights", wts, 4, 3, d);
    char a[] = "data";
    return read_ProjWeightData(a, projections, weights, datafile_row0, proj_rows, proj_cols, proj_start, proj_num,
                               sink());
}

int ref_gen_views(float *views, float *times, int K, int N_theta, int proj_start, int N_p, float min_acq_time,
                  float rot_speed)
{
    return gen_interlaced_views_0_to_Inf(views, times, K, N_theta, proj_start, N_p, min_acq_time, rot_speed,
                                         sink());
}
