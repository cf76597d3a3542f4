/*
 * vs_frameinfo.c -- frame geometry and host frame buffers (the API of
 * src/frameinfo.h:84-120 of the reference, same semantics).
 */
#include <string.h>

#include "vidstab_b200.h"

int vsFrameInfoInit(VSFrameInfo* fi, int width, int height, VSPixelFormat pFormat) {
  fi->pFormat = pFormat;
  fi->width = width;
  fi->height = height;
  fi->planes = 3;
  fi->log2ChromaW = 0;
  fi->log2ChromaH = 0;
  fi->bytesPerPixel = 1;
  switch (pFormat) {
    case PF_GRAY8: fi->planes = 1; break;
    case PF_YUV420P: fi->log2ChromaW = 1; fi->log2ChromaH = 1; break;
    case PF_YUV422P: fi->log2ChromaW = 1; break;
    case PF_YUV444P: break;
    case PF_YUV410P: fi->log2ChromaW = 2; fi->log2ChromaH = 2; break;
    case PF_YUV411P: fi->log2ChromaW = 2; break;
    case PF_YUV440P: fi->log2ChromaH = 1; break;
    case PF_YUVA420P: fi->log2ChromaW = 1; fi->log2ChromaH = 1; fi->planes = 4; break;
    case PF_RGB24:
    case PF_BGR24: fi->bytesPerPixel = 3; fi->planes = 1; break;
    case PF_RGBA: fi->bytesPerPixel = 4; fi->planes = 1; break;
    default: fi->pFormat = 0; return 0;
  }
  if (width <= 0 || height <= 0) {
    vs_log_error("vid.stab", "invalid frame dimensions %ix%i: width and height must be positive\n",
                 width, height);
    fi->pFormat = 0;
    return 0;
  }
  if (width % (1 << fi->log2ChromaW) != 0 || height % (1 << fi->log2ChromaH) != 0) {
    vs_log_error("vid.stab",
                 "invalid frame dimensions %ix%i for pixel format %i: the chroma "
                 "subsampling needs multiples of %i (width) and %i (height)\n",
                 width, height, (int)pFormat, 1 << fi->log2ChromaW, 1 << fi->log2ChromaH);
    fi->pFormat = 0;
    return 0;
  }
  return 1;
}

int vsGetPlaneWidthSubS(const VSFrameInfo* fi, int plane) {
  return (plane == 1 || plane == 2) ? fi->log2ChromaW : 0;
}

int vsGetPlaneHeightSubS(const VSFrameInfo* fi, int plane) {
  return (plane == 1 || plane == 2) ? fi->log2ChromaH : 0;
}

int vsFrameIsNull(const VSFrame* frame) { return frame == 0 || frame->data[0] == 0; }

int vsFramesEqual(const VSFrame* a, const VSFrame* b) {
  return a && b && (a == b || a->data[0] == b->data[0]);
}

void vsFrameNull(VSFrame* frame) {
  memset(frame->data, 0, sizeof(frame->data));
  memset(frame->linesize, 0, sizeof(frame->linesize));
}

void vsFrameAllocate(VSFrame* frame, const VSFrameInfo* fi) {
  vsFrameNull(frame);
  if (fi->pFormat < PF_PACKED) {
    for (int p = 0; p < fi->planes && p < 4; p++) {
      int w = fi->width >> vsGetPlaneWidthSubS(fi, p);
      int h = fi->height >> vsGetPlaneHeightSubS(fi, p);
      frame->data[p] = (uint8_t*)vs_zalloc((size_t)w * h);
      frame->linesize[p] = w;
      if (!frame->data[p]) vs_log_error("vid.stab", "out of memory: cannot allocate a frame plane");
    }
  } else {
    frame->data[0] = (uint8_t*)vs_zalloc((size_t)fi->width * fi->height * fi->bytesPerPixel);
    frame->linesize[0] = fi->width * fi->bytesPerPixel;
    if (!frame->data[0]) vs_log_error("vid.stab", "out of memory: cannot allocate a frame");
  }
}

void vsFrameCopyPlane(VSFrame* dest, const VSFrame* src, const VSFrameInfo* fi, int plane) {
  int h = fi->height >> vsGetPlaneHeightSubS(fi, plane);
  if (src->linesize[plane] == dest->linesize[plane]) {
    memcpy(dest->data[plane], src->data[plane], (size_t)src->linesize[plane] * h);
    return;
  }
  int rowbytes = (fi->width >> vsGetPlaneWidthSubS(fi, plane)) * fi->bytesPerPixel;
  uint8_t* d = dest->data[plane];
  const uint8_t* s = src->data[plane];
  for (int r = 0; r < h; r++) {
    memcpy(d, s, (size_t)rowbytes);
    d += dest->linesize[plane];
    s += src->linesize[plane];
  }
}

void vsFrameCopy(VSFrame* dest, const VSFrame* src, const VSFrameInfo* fi) {
  for (int p = 0; p < fi->planes && p < 4; p++) vsFrameCopyPlane(dest, src, fi, p);
}

void vsFrameFillFromBuffer(VSFrame* frame, uint8_t* img, const VSFrameInfo* fi) {
  vsFrameNull(frame);
  size_t off = 0;
  for (int p = 0; p < fi->planes && p < 4; p++) {
    int w = fi->width >> vsGetPlaneWidthSubS(fi, p);
    int h = fi->height >> vsGetPlaneHeightSubS(fi, p);
    frame->data[p] = img + off;
    frame->linesize[p] = w * fi->bytesPerPixel;
    off += (size_t)h * w * fi->bytesPerPixel;
  }
}

void vsFrameFree(VSFrame* frame) {
  for (int p = 0; p < 4; p++) {
    if (frame->data[p]) vs_free(frame->data[p]);
    frame->data[p] = 0;
    frame->linesize[p] = 0;
  }
}
