/*
 * vs_pnet.c -- entry points of the learned search proposal (declared in
 * vidstab_b200_ext.h).  No counterpart in the reference: the reference
 * searches every field over its whole lattice (src/motiondetect.c:439-586);
 * a detector with a proposal narrows that search and falls back to it.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "vidstab_b200.h"
#include "vidstab_b200_ext.h"
#include "vsb_host.h"

/* header of a serialized network ("VSBP" file), followed by the bf16
   weights and the f32 biases in device-buffer order */
typedef struct {
  char magic[4];
  int32_t version;
  int32_t n_bf16;
  int32_t n_f32;
  float scale;       /* network units -> pixels */
  float radius;      /* pixels around the prediction */
  float conf_min;    /* confidence logit threshold */
  float match_bound; /* trusted refined SAD per field pixel */
} pnet_header;

#define PNET_NB16 30208
#define PNET_NF32 131

int vsb_pnet_sizes(long* n_bf16, long* n_f32, long* act_bytes_per_item,
                   long* work_bytes_per_item) {
  if (n_bf16) *n_bf16 = PNET_NB16;
  if (n_f32) *n_f32 = PNET_NF32;
  if (act_bytes_per_item) *act_bytes_per_item = 2L * (32768 + 8192 + 2048 + 512);
  if (work_bytes_per_item) *work_bytes_per_item = 4L * (32768 + 8192 + 2048 + 512);
  return vsbd_pnet_param_bytes() == 2L * PNET_NB16 + 4L * PNET_NF32 ? VS_OK : VS_ERROR;
}

int vsb_pnet_parse(const void* blob, long bytes, double radius, double conf_min,
                   double match_bound, vsb_pnet_settings* out) {
  pnet_header h;
  if (bytes < (long)sizeof(h)) {
    vsbd_set_error("proposal network: blob shorter than its header");
    return VS_ERROR;
  }
  memcpy(&h, blob, sizeof(h));
  if (memcmp(h.magic, "VSBP", 4) != 0 || h.version != 1 || h.n_bf16 != PNET_NB16 ||
      h.n_f32 != PNET_NF32 || bytes != (long)sizeof(h) + vsbd_pnet_param_bytes()) {
    vsbd_set_error("proposal network: not a version-1 VSBP blob of this architecture");
    return VS_ERROR;
  }
  out->params = (const char*)blob + sizeof(h);
  out->scale = h.scale;
  out->radius = (float)(radius >= 0 ? radius : h.radius);
  out->conf_min = (float)(isnan(conf_min) ? h.conf_min : conf_min);
  out->match_bound = (float)(match_bound >= 0 ? match_bound : h.match_bound);
  return VS_OK;
}

int vsb_set_proposal_ex(VSMotionDetect* md, const void* blob, long bytes, double radius,
                        double conf_min, double match_bound) {
  vsbd_ctx* c = vsb_md_device(md);
  if (!c) {
    vsbd_set_error("detector has no device state (not initialised)");
    return VS_ERROR;
  }
  if (!blob) return vsbd_set_proposal(c, NULL, 0, 0, 0, 0) == 0 ? VS_OK : VS_ERROR;
  vsb_pnet_settings p;
  if (vsb_pnet_parse(blob, bytes, radius, conf_min, match_bound, &p) != VS_OK) return VS_ERROR;
  /* very shaky footage (shakiness >= 8): the second pass around the global
     model keeps large motions inside the network's reach */
  if (vsbd_set_proposal_passes(c, md->conf.shakiness >= 8 ? 2 : 1) != 0) return VS_ERROR;
  return vsbd_set_proposal(c, p.params, p.scale, p.radius, p.conf_min, p.match_bound) == 0
             ? VS_OK
             : VS_ERROR;
}

int vsb_set_proposal(VSMotionDetect* md, const void* blob, long bytes) {
  return vsb_set_proposal_ex(md, blob, bytes, -1.0, NAN, -1.0);
}

int vsb_set_proposal_scope(VSMotionDetect* md, int fine_net, double fine_radius) {
  return vsbd_set_proposal_scope(vsb_md_device(md), fine_net, (float)fine_radius) == 0 ? VS_OK
                                                                                       : VS_ERROR;
}

int vsb_set_proposal_passes(VSMotionDetect* md, int passes) {
  return vsbd_set_proposal_passes(vsb_md_device(md), passes) == 0 ? VS_OK : VS_ERROR;
}

int vsb_set_proposal_verify(VSMotionDetect* md, int on) {
  return vsbd_set_proposal_verify(vsb_md_device(md), on) == 0 ? VS_OK : VS_ERROR;
}

int vsb_proposal_stats(const VSMotionDetect* md, long long* stats) {
  return vsbd_proposal_stats(vsb_md_device(md), stats) == 0 ? VS_OK : VS_ERROR;
}

int vsb_set_field_log(VSMotionDetect* md, void* d_inputs, void* d_labels, long cap) {
  return vsbd_set_field_log(vsb_md_device(md), d_inputs, d_labels, cap) == 0 ? VS_OK : VS_ERROR;
}

long vsb_field_log_count(const VSMotionDetect* md) {
  return vsbd_field_log_count(vsb_md_device(md));
}

int vsb_pnet_forward_train(const void* d_params, const void* d_input, int n, void* d_acts,
                           float* d_out, void* stream) {
  return vsbd_pnet_forward_train(d_params, d_input, n, d_acts, d_out, stream) == 0 ? VS_OK
                                                                                   : VS_ERROR;
}

int vsb_pnet_backward(const void* d_params, const void* d_input, const void* d_acts, int n,
                      const float* d_dout, float* d_grad, void* d_work, void* stream) {
  return vsbd_pnet_backward(d_params, d_input, d_acts, n, d_dout, d_grad, d_work, stream) == 0
             ? VS_OK
             : VS_ERROR;
}

int vsb_pnet_infer(const void* d_params, const void* d_input, int n, float* d_out, void* stream) {
  return vsbd_pnet_infer(d_params, d_input, n, d_out, stream) == 0 ? VS_OK : VS_ERROR;
}

int vsb_pnet_infer_items(const void* d_params, const uint8_t* d_curr, const uint8_t* d_prev,
                         int pitch, int width, int height, const void* d_items, int n,
                         float* d_out, void* stream) {
  return vsbd_pnet_infer_items(d_params, d_curr, d_prev, pitch, width, height, d_items, n, d_out,
                               stream) == 0
             ? VS_OK
             : VS_ERROR;
}

int vsb_pnet_crops(const uint8_t* d_curr, const uint8_t* d_prev, int pitch, int width, int height,
                   const void* d_items, int n, void* d_input, void* stream) {
  return vsbd_pnet_crops(d_curr, d_prev, pitch, width, height, d_items, n, d_input, stream) == 0
             ? VS_OK
             : VS_ERROR;
}

int vsb_pnet_narrow_host(const uint8_t* curr, const uint8_t* prev, int width, int height,
                         int size, int maxShift, int stepSize, const int16_t* x, const int16_t* y,
                         const int16_t* ox, const int16_t* oy, int n, const float* pout,
                         float scale, float radius, float conf_min, uint32_t sad_bound,
                         uint32_t* sad, int16_t* tx, int16_t* ty, int32_t* ok, uint8_t* flags) {
  vsbd_geom g;
  int32_t* order = NULL;
  if (vsb_build_geom(&g, &order, size, 1, maxShift, stepSize, 1) != 0) return VS_ERROR;
  vsbd_item* items = (vsbd_item*)malloc(sizeof(vsbd_item) * (size_t)(n > 0 ? n : 1));
  vsbd_result* res = (vsbd_result*)malloc(sizeof(vsbd_result) * (size_t)(n > 0 ? n : 1));
  for (int i = 0; i < n; i++) {
    items[i].x = x[i];
    items[i].y = y[i];
    items[i].ox = ox ? ox[i] : 0;
    items[i].oy = oy ? oy[i] : 0;
  }
  int rc = n > 0 ? vsbd_pnet_narrow_host(curr, prev, width, height, &g, items, n, pout, scale,
                                         radius, conf_min, sad_bound, res, flags)
                 : 0;
  for (int i = 0; rc == 0 && i < n; i++) {
    sad[i] = res[i].sad;
    tx[i] = res[i].tx;
    ty[i] = res[i].ty;
    ok[i] = res[i].ok;
  }
  free(items);
  free(res);
  free(order);
  return rc == 0 ? VS_OK : VS_ERROR;
}
