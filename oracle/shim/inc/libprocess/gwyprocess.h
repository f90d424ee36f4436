/* gwyprocess.h -- the GwyDataField / GwyDataLine subset used by GSvit's CPU
 * solver files, as plain heap arrays of doubles.  Test infrastructure only. */
#ifndef SHIM_GWYPROCESS_H
#define SHIM_GWYPROCESS_H
#include <glib.h>

typedef enum { GWY_INTERPOLATION_NONE = 0, GWY_INTERPOLATION_ROUND = 1, GWY_INTERPOLATION_LINEAR = 2 } GwyInterpolationType;

typedef struct _GwyDataField { gint xres, yres; gdouble xreal, yreal; gdouble *data; } GwyDataField;
typedef struct _GwyDataLine { gint res; gdouble real; gdouble *data; } GwyDataLine;
typedef struct _GwyBrick { gint xres, yres, zres; gdouble *data; } GwyBrick;
typedef struct _GwySIUnit { gint dummy; } GwySIUnit;

static inline GwyDataField *gwy_data_field_new(gint xres, gint yres, gdouble xreal, gdouble yreal, gboolean nullme)
{
    GwyDataField *f = (GwyDataField *)g_malloc(sizeof(GwyDataField));
    f->xres = xres; f->yres = yres; f->xreal = xreal; f->yreal = yreal;
    f->data = (gdouble *)(nullme ? g_malloc0(sizeof(gdouble) * (gsize)xres * (gsize)yres)
                                 : g_malloc(sizeof(gdouble) * (gsize)xres * (gsize)yres));
    (void)nullme;
    return f;
}
static inline gint gwy_data_field_get_xres(GwyDataField *f) { return f->xres; }
static inline gint gwy_data_field_get_yres(GwyDataField *f) { return f->yres; }
static inline gdouble *gwy_data_field_get_data(GwyDataField *f) { return f->data; }
static inline gdouble gwy_data_field_get_val(GwyDataField *f, gint col, gint row) { return f->data[(gsize)row * f->xres + col]; }
static inline void gwy_data_field_set_val(GwyDataField *f, gint col, gint row, gdouble v) { f->data[(gsize)row * f->xres + col] = v; }
static inline void gwy_data_field_resample(GwyDataField *f, gint xres, gint yres, GwyInterpolationType it)
{
    (void)it;
    if (xres == f->xres && yres == f->yres) return;
    g_free(f->data);
    f->xres = xres; f->yres = yres;
    f->data = (gdouble *)g_malloc0(sizeof(gdouble) * (gsize)xres * (gsize)yres);
}
static inline void gwy_data_field_data_changed(GwyDataField *f) { (void)f; }

static inline GwyDataLine *gwy_data_line_new(gint res, gdouble real, gboolean nullme)
{
    GwyDataLine *l = (GwyDataLine *)g_malloc(sizeof(GwyDataLine));
    l->res = res; l->real = real;
    l->data = (gdouble *)g_malloc0(sizeof(gdouble) * (gsize)(res > 0 ? res : 1));
    (void)nullme;
    return l;
}
static inline gint gwy_data_line_get_res(GwyDataLine *l) { return l->res; }
static inline void gwy_data_line_set_val(GwyDataLine *l, gint i, gdouble v) { l->data[i] = v; }
static inline void gwy_data_line_resample(GwyDataLine *l, gint res, GwyInterpolationType it)
{
    (void)it;
    if (res == l->res) return;
    g_free(l->data);
    l->res = res;
    l->data = (gdouble *)g_malloc0(sizeof(gdouble) * (gsize)res);
}
#endif
