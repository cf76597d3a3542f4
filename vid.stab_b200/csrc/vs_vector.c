/*
 * vs_vector.c -- the growable pointer vector LocalMotions is built on and
 * the small double array (the API of src/vsvector.h:35-222 of the
 * reference, same semantics: elements are owned pointers, the vector never
 * shrinks, set() grows to any valid position).
 */
#include <string.h>

#include "vidstab_b200.h"
#include "vsb_host.h"

static int grow_to(VSVector* V, int newsize) {
  if (newsize < 1) newsize = 1;
  void** d = (void**)vs_realloc(V->data, (size_t)newsize * sizeof(void*));
  if (!d) {
    vsb_note_oom();
    vs_log_error("VS_Vector", "out of memory!");
    return VS_ERROR;
  }
  V->data = d;
  V->buffersize = newsize;
  if (V->nelems > V->buffersize) V->nelems = V->buffersize;
  return VS_OK;
}

int vs_vector_init(VSVector* V, int buffersize) {
  if (buffersize > 0) {
    V->data = (void**)vs_zalloc(sizeof(void*) * (size_t)buffersize);
    if (!V->data) {
      vsb_note_oom();
      V->buffersize = V->nelems = 0;
      return VS_ERROR;
    }
  } else {
    V->data = 0;
    buffersize = 0;
  }
  V->buffersize = buffersize;
  V->nelems = 0;
  return VS_OK;
}

int vs_vector_fini(VSVector* V) {
  if (V->data) vs_free(V->data);
  V->data = 0;
  V->buffersize = 0;
  V->nelems = 0;
  return VS_OK;
}

int vs_vector_zero(VSVector* V) {
  for (int i = 0; i < V->nelems; i++)
    if (V->data[i]) vs_free(V->data[i]);
  V->nelems = 0;
  return VS_OK;
}

int vs_vector_del(VSVector* V) {
  vs_vector_zero(V);
  return vs_vector_fini(V);
}

int vs_vector_size(const VSVector* V) { return V->nelems; }

int vs_vector_append(VSVector* V, void* data) {
  if (!V->data || V->buffersize < 1) {
    if (vs_vector_init(V, 4) != VS_OK) return VS_ERROR;
  }
  if (V->nelems >= V->buffersize) {
    if (grow_to(V, V->buffersize * 2) != VS_OK) return VS_ERROR;
  }
  V->data[V->nelems++] = data;
  return VS_OK;
}

int vs_vector_append_dup(VSVector* V, void* data, int data_size) {
  void* d = vs_malloc((size_t)data_size);
  if (!d) {
    vsb_note_oom();
    return VS_ERROR;
  }
  memcpy(d, data, (size_t)data_size);
  if (vs_vector_append(V, d) != VS_OK) {
    vs_free(d);
    return VS_ERROR;
  }
  return VS_OK;
}

void* vs_vector_get(const VSVector* V, int pos) {
  if (pos < 0 || pos >= V->nelems) return 0;
  return V->data[pos];
}

int vs_vector_set(VSVector* V, int pos, void* data, void** old) {
  if (old) *old = 0;
  if (pos < 0 || pos >= VS_VECTOR_MAX_SIZE) {
    vs_log_error("VS_Vector", "position %i out of range [0,%i)!", pos, VS_VECTOR_MAX_SIZE);
    return VS_ERROR;
  }
  if (!V->data || V->buffersize < 1) {
    if (vs_vector_init(V, 4) != VS_OK) return VS_ERROR;
  }
  if (V->buffersize <= pos) {
    int n = V->buffersize;
    while (n <= pos && n <= VS_VECTOR_MAX_SIZE / 2) n *= 2;
    if (n <= pos) n = pos + 1;
    if (grow_to(V, n) != VS_OK) return VS_ERROR;
  }
  for (int i = V->nelems; i <= pos; i++) V->data[i] = 0;
  if (pos >= V->nelems) V->nelems = pos + 1;
  if (old) *old = V->data[pos];
  V->data[pos] = data;
  return VS_OK;
}

int vs_vector_set_dup(VSVector* V, int pos, void* data, int data_size, void** old) {
  if (old) *old = 0;
  void* d = vs_malloc((size_t)data_size);
  if (!d) {
    vsb_note_oom();
    return VS_ERROR;
  }
  memcpy(d, data, (size_t)data_size);
  int rc = vs_vector_set(V, pos, d, old);
  if (rc != VS_OK) vs_free(d);
  return rc;
}

VSVector vs_vector_filter(const VSVector* V, short (*pred)(void*, void*), void* param) {
  VSVector r;
  vs_vector_init(&r, V->nelems);
  for (int i = 0; i < V->nelems; i++)
    if (pred(param, V->data[i])) vs_vector_append(&r, V->data[i]);
  return r;
}

VSVector vs_vector_concat(const VSVector* V1, const VSVector* V2) {
  VSVector r;
  if (vs_vector_init(&r, V1->nelems + V2->nelems) != VS_OK) return r; /* empty, no data */
  if (V1->nelems) memcpy(r.data, V1->data, sizeof(void*) * (size_t)V1->nelems);
  if (V2->nelems) memcpy(r.data + V1->nelems, V2->data, sizeof(void*) * (size_t)V2->nelems);
  r.nelems = V1->nelems + V2->nelems;
  return r;
}

VSArray vs_array_new(int len) {
  VSArray a;
  a.dat = (double*)vs_zalloc(sizeof(double) * (size_t)(len > 0 ? len : 1));
  a.len = a.dat ? len : 0;
  if (!a.dat) vsb_note_oom();
  return a;
}

VSArray vs_array(double vals[], int len) {
  VSArray a = vs_array_new(len);
  if (len > 0) memcpy(a.dat, vals, sizeof(double) * (size_t)len);
  return a;
}

VSArray* vs_array_plus(VSArray* c, VSArray a, VSArray b) {
  if (c->len == 0) *c = vs_array_new(a.len);
  for (int i = 0; i < a.len && i < b.len; i++) c->dat[i] = a.dat[i] + b.dat[i];
  return c;
}

VSArray* vs_array_scale(VSArray* c, VSArray a, double f) {
  if (c->len == 0) *c = vs_array_new(a.len);
  for (int i = 0; i < a.len; i++) c->dat[i] = a.dat[i] * f;
  return c;
}

VSArray vs_array_copy(VSArray a) {
  VSArray c = vs_array_new(a.len);
  if (a.len > 0) memcpy(c.dat, a.dat, sizeof(double) * (size_t)a.len);
  return c;
}

void vs_array_zero(VSArray* a) {
  if (a->len > 0) memset(a->dat, 0, sizeof(double) * (size_t)a->len);
}

void vs_array_swap(VSArray* a, VSArray* b) {
  VSArray t = *a;
  *a = *b;
  *b = t;
}

void vs_array_free(VSArray a) { vs_free(a.dat); }

void vs_array_print(VSArray a, FILE* f) {
  for (int i = 0; i < a.len; i++) fprintf(f, "%g ", a.dat[i]);
}
