/*
 * vs_draw.c -- the `show` overlay: field boxes, scan areas and shift lines
 * drawn into the caller's frame (src/motiondetect.c:813-952 of the
 * reference, same pixels).  Planar formats draw into the luma plane, packed
 * formats into every colour channel (alpha untouched).  Built with the
 * reference build's floating-point flags because line positions are
 * truncated from doubles.
 *
 * The shift line starts at the field centre through a Vec* that aliases the
 * motion's Field, and a line drawn right-to-left or bottom-to-top moves that
 * start point to the end point -- which rewrites the returned motion's field
 * position, as the reference does.  Kept so that show != 0 returns the same
 * LocalMotions.
 */
#include <math.h>
#include <stdlib.h>

#include "vidstab_b200.h"
#include "vsb_host.h"

static void hline(uint8_t* I, int ls, int w, int h, int bpp, int x, int y, int len, uint8_t col) {
  if (y < 0 || y >= h || len <= 0) return;
  if (x < 0) { len += x; x = 0; }
  if (x + len > w) len = w - x;
  if (len <= 0) return;
  int ch = bpp > 3 ? 3 : bpp;
  uint8_t* p = I + (long)x * bpp + (long)y * ls;
  for (int k = 0; k < len; k++, p += bpp)
    for (int c = 0; c < ch; c++) p[c] = col;
}

static void vline(uint8_t* I, int ls, int w, int h, int bpp, int x, int y, int len, uint8_t col) {
  if (x < 0 || x >= w || len <= 0) return;
  if (y < 0) { len += y; y = 0; }
  if (y + len > h) len = h - y;
  if (len <= 0) return;
  int ch = bpp > 3 ? 3 : bpp;
  uint8_t* p = I + (long)x * bpp + (long)y * ls;
  for (int k = 0; k < len; k++, p += ls)
    for (int c = 0; c < ch; c++) p[c] = col;
}

static void box(uint8_t* I, int ls, int w, int h, int bpp, int x, int y, int sx, int sy, uint8_t col) {
  for (int j = 0; j < sy; j++) hline(I, ls, w, h, bpp, x - sx / 2, y - sy / 2 + j, sx, col);
}

static void rect(uint8_t* I, int ls, int w, int h, int bpp, int x, int y, int sx, int sy, uint8_t col) {
  hline(I, ls, w, h, bpp, x - sx / 2, y - sy / 2, sx, col);
  hline(I, ls, w, h, bpp, x - sx / 2, y + sy / 2, sx, col);
  vline(I, ls, w, h, bpp, x - sx / 2, y - sy / 2, sy, col);
  vline(I, ls, w, h, bpp, x + sx / 2, y - sy / 2, sy, col);
}

static void line(uint8_t* I, int ls, int w, int h, int bpp, Vec* a, Vec* b, int thickness, uint8_t col) {
  Vec div = sub_vec(*b, *a);
  if (div.y == 0) {
    if (div.x < 0) { *a = *b; div.x *= -1; }
    for (int r = -thickness / 2; r <= thickness / 2; r++)
      hline(I, ls, w, h, bpp, a->x, a->y + r, div.x + 1, col);
  } else if (div.x == 0) {
    if (div.y < 0) { *a = *b; div.y *= -1; }
    for (int r = -thickness / 2; r <= thickness / 2; r++)
      vline(I, ls, w, h, bpp, a->x + r, a->y, div.y + 1, col);
  } else {
    double m = (double)div.x / (double)div.y;
    int horlen = thickness + fabs(m);
    for (int c = 0; c <= abs(div.y); c++) {
      int dy = div.y < 0 ? -c : c;
      int x = a->x + m * dy - horlen / 2;
      hline(I, ls, w, h, bpp, x, a->y + dy, horlen + 1, col);
    }
  }
}

void vsb_draw_motions(VSMotionDetect* md, LocalMotions* coarse, LocalMotions* fine) {
  uint8_t* I = md->currorig.data[0];
  if (!I) return;
  int ls = md->currorig.linesize[0];
  int w = md->fi.width, h = md->fi.height;
  int bpp = md->fi.pFormat > PF_PACKED ? md->fi.bytesPerPixel : 1;
  int nc = vs_vector_size(coarse), nf = vs_vector_size(fine);
  int maxShift = md->fieldscoarse.maxShift;
  if (md->conf.show > 1)
    for (int i = 0; i < nc; i++) {
      LocalMotion* lm = LMGet(coarse, i);
      rect(I, ls, w, h, bpp, lm->f.x, lm->f.y, lm->f.size + 2 * maxShift, lm->f.size + 2 * maxShift, 80);
    }
  for (int i = 0; i < nc; i++) {
    LocalMotion* lm = LMGet(coarse, i);
    box(I, ls, w, h, bpp, lm->f.x, lm->f.y, lm->f.size, lm->f.size, 40);
  }
  for (int i = 0; i < nf; i++) {
    LocalMotion* lm = LMGet(fine, i);
    rect(I, ls, w, h, bpp, lm->f.x, lm->f.y, lm->f.size, lm->f.size, 40);
  }
  for (int k = 0; k < 2; k++) {
    LocalMotions* v = k == 0 ? coarse : fine;
    uint8_t col = k == 0 ? 180 : 64;
    int n = vs_vector_size(v);
    for (int i = 0; i < n; i++) {
      LocalMotion* lm = LMGet(v, i);
      Vec end = add_vec(field_to_vec(lm->f), lm->v);
      box(I, ls, w, h, bpp, lm->f.x, lm->f.y, 5, 5, 0);
      box(I, ls, w, h, bpp, lm->f.x + lm->v.x, lm->f.y + lm->v.y, 5, 5, 250);
      line(I, ls, w, h, bpp, (Vec*)&lm->f, &end, 3, col);
    }
  }
}
