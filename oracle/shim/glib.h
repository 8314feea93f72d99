/* Minimal stand-in for the few GLib declarations that Obit's vector-math
 * sources (ObitSinCos.c, ObitExp.c, ObitVecFunc.c), its GPU sky-model host glue
 * (ObitGPUSkyModel.c) and the headers they pull in (Obit.h, ObitTypes.h,
 * ObitErr.h, ObitInfoList.h, ObitThread.h, ObitUV.h, ObitSkyModel.h ...) need
 * at compile time.  Only used to build the reference-derived test libraries
 * under _ref/; nothing in the product includes it. */
#ifndef OBIT_ORACLE_GLIB_SHIM_H
#define OBIT_ORACLE_GLIB_SHIM_H
#include <stddef.h>
#include <stdarg.h>
typedef char gchar;
typedef unsigned char guchar;
typedef short gshort;
typedef unsigned short gushort;
typedef int gint;
typedef unsigned int guint;
typedef long glong;
typedef unsigned long gulong;
typedef int gint32;
typedef unsigned int guint32;
typedef short gint16;
typedef unsigned short guint16;
typedef signed char gint8;
typedef unsigned char guint8;
typedef long long gint64;
typedef unsigned long long guint64;
typedef float gfloat;
typedef double gdouble;
typedef int gboolean;
typedef void *gpointer;
typedef const void *gconstpointer;
typedef size_t gsize;
typedef struct _GSList { gpointer data; struct _GSList *next; } GSList;
typedef struct _GQueue GQueue;
typedef struct _GMutex GMutex;
typedef struct _GCond GCond;
typedef struct _GThread GThread;
typedef struct _GThreadPool GThreadPool;
typedef struct _GAsyncQueue GAsyncQueue;
typedef struct _GHashTable GHashTable;
typedef struct _GString GString;
#ifndef FALSE
#define FALSE 0
#endif
#ifndef TRUE
#define TRUE 1
#endif
#define G_PI 3.1415926535897932384626433832795028841971693993751
#ifndef MAX
#define MAX(a, b) (((a) > (b)) ? (a) : (b))
#endif
#ifndef MIN
#define MIN(a, b) (((a) < (b)) ? (a) : (b))
#endif
#define G_STMT_START do
#define G_STMT_END while (0)
#define G_GNUC_PRINTF(a, b)
void g_error(const gchar *fmt, ...);
gpointer g_malloc0(gsize n);
void g_free(gpointer p);
gchar *g_strdup(const gchar *s);
typedef gpointer (*GThreadFunc)(gpointer data);
#define g_assert(e) ((void)0)
gchar *g_strconcat(const gchar *s, ...);
gint g_snprintf(gchar *s, gulong n, const gchar *fmt, ...);
#endif
