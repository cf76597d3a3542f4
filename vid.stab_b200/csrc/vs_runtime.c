/*
 * vs_runtime.c -- pluggable allocation and logging hooks and the return
 * codes of the public API (the counterpart of src/libvidstab.c:33-75 of the
 * reference).  Hosts such as ffmpeg replace vs_log / vs_malloc / ... with
 * their own functions; the library calls only through these pointers.
 */
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "vidstab_b200.h"

static void* zalloc_default(size_t size) {
  void* p = malloc(size);
  if (p) memset(p, 0, size);
  return p;
}

static int log_default(int type, const char* tag, const char* format, ...) {
  if (vs_log_level < type) return 0;
  const char* kind = type == VS_ERROR_TYPE  ? "Error: "
                     : type == VS_WARN_TYPE ? "Warn:  "
                     : type == VS_INFO_TYPE ? "Info:  "
                     : type == VS_MSG_TYPE  ? "Msg:   "
                                            : "Unknown";
  fprintf(stderr, "%s (%s):", kind, tag ? tag : "");
  va_list ap;
  va_start(ap, format);
  vfprintf(stderr, format, ap);
  va_end(ap);
  fputc('\n', stderr);
  return 0;
}

vs_malloc_t vs_malloc = malloc;
vs_realloc_t vs_realloc = realloc;
vs_free_t vs_free = free;
vs_zalloc_t vs_zalloc = zalloc_default;
vs_strdup_t vs_strdup = strdup;
vs_log_t vs_log = log_default;

int VS_ERROR_TYPE = 0;
int VS_WARN_TYPE = 1;
int VS_INFO_TYPE = 2;
int VS_MSG_TYPE = 3;

int VS_ERROR = -1;
int VS_OK = 0;

int vs_log_level = 4;

/* allocation failures through the hooks above, counted per thread: the
   detect path compares the count before and after a frame's host work and
   fails the frame (VS_ERROR) when it moved, whatever helper met the failure */
static __thread int g_oom;
void vsb_note_oom(void) { g_oom++; }
int vsb_oom_count(void) { return g_oom; }
