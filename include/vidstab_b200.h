/*
 * vidstab_b200.h -- public C ABI of the B200 motion-detection library.
 *
 * The library is a drop-in for the detect half of vid.stab (the work behind
 * ffmpeg's `vidstabdetect`).  Every type below has the same name, member
 * order and size as the reference's, and every function the same name,
 * signature, argument meaning and return convention, so that a caller built
 * against the reference headers links against libvidstab_b200.so unchanged.
 * The reference interface each declaration replaces is cited beside it
 * (paths relative to the vid.stab source tree).
 *
 * The per-frame detect (vsMotionDetection) runs on one NVIDIA B200 GPU; there
 * is no CPU fallback: without a usable CUDA device vsMotionDetectInit fails
 * with VS_ERROR and logs why.
 *
 * Entry points with the vsb_ prefix have no counterpart in the reference;
 * they are declared in vidstab_b200_ext.h.
 */
#ifndef VIDSTAB_B200_H
#define VIDSTAB_B200_H

#include <stddef.h>
#include <stdint.h>
#include <stdio.h>

#if defined(__GNUC__) && __GNUC__ >= 4
#define VS_API __attribute__((visibility("default")))
#else
#define VS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- runtime services: src/vidstabdefines.h:84-117, src/libvidstab.c:59-75 */
typedef void* (*vs_malloc_t)(size_t size);
typedef void* (*vs_realloc_t)(void* ptr, size_t size);
typedef void (*vs_free_t)(void* ptr);
typedef void* (*vs_zalloc_t)(size_t size);
typedef int (*vs_log_t)(int type, const char* tag, const char* format, ...);
typedef char* (*vs_strdup_t)(const char* s);

extern VS_API vs_log_t vs_log;           /* replaces src/vidstabdefines.h:93 */
extern VS_API int vs_log_level;          /* :94 */
extern VS_API vs_malloc_t vs_malloc;     /* :96 */
extern VS_API vs_realloc_t vs_realloc;   /* :97 */
extern VS_API vs_free_t vs_free;         /* :98 */
extern VS_API vs_zalloc_t vs_zalloc;     /* :99 */
extern VS_API vs_strdup_t vs_strdup;     /* :101 */
extern VS_API int VS_ERROR_TYPE;         /* :103-106 */
extern VS_API int VS_WARN_TYPE;
extern VS_API int VS_INFO_TYPE;
extern VS_API int VS_MSG_TYPE;
extern VS_API int VS_ERROR;              /* :108, value -1 */
extern VS_API int VS_OK;                 /* :109, value 0 */

#define vs_log_error(...) vs_log(VS_ERROR_TYPE, __VA_ARGS__)
#define vs_log_warn(...) vs_log(VS_WARN_TYPE, __VA_ARGS__)
#define vs_log_info(...) vs_log(VS_INFO_TYPE, __VA_ARGS__)
#define vs_log_msg(...) vs_log(VS_MSG_TYPE, __VA_ARGS__)

#define VS_MAX(a, b) (((a) > (b)) ? (a) : (b))
#define VS_MIN(a, b) (((a) < (b)) ? (a) : (b))
#define VS_CLAMP(x, a, b) VS_MIN(VS_MAX((a), (x)), (b))

/* ---- frames: src/frameinfo.h:34-67 --------------------------------------- */
typedef enum {
  PF_NONE = -1,
  PF_GRAY8,
  PF_YUV420P,
  PF_YUV422P,
  PF_YUV444P,
  PF_YUV410P,
  PF_YUV411P,
  PF_YUV440P,
  PF_YUVA420P,
  PF_PACKED, /* marker: packed formats follow */
  PF_RGB24,
  PF_BGR24,
  PF_RGBA,
  PF_NUMBER
} VSPixelFormat;

typedef struct vsframeinfo {
  int width, height;
  int planes;
  int log2ChromaW;
  int log2ChromaH;
  VSPixelFormat pFormat;
  int bytesPerPixel;
} VSFrameInfo;

/* plane pointers and row distances in BYTES (ffmpeg's AVFrame convention) */
typedef struct vsframe {
  uint8_t* data[4];
  int linesize[4];
} VSFrame;

VS_API int vsFrameInfoInit(VSFrameInfo* fi, int width, int height, VSPixelFormat pFormat); /* src/frameinfo.h:84 */
VS_API int vsGetPlaneWidthSubS(const VSFrameInfo* fi, int plane);      /* :88 */
VS_API int vsGetPlaneHeightSubS(const VSFrameInfo* fi, int plane);     /* :91 */
VS_API void vsFrameNull(VSFrame* frame);                               /* :94 */
VS_API int vsFrameIsNull(const VSFrame* frame);                        /* :97 */
VS_API int vsFramesEqual(const VSFrame* frame1, const VSFrame* frame2); /* :100 */
VS_API void vsFrameAllocate(VSFrame* frame, const VSFrameInfo* fi);    /* :103 */
VS_API void vsFrameCopyPlane(VSFrame* dest, const VSFrame* src, const VSFrameInfo* fi,
                             int plane);                               /* :107 */
VS_API void vsFrameCopy(VSFrame* dest, const VSFrame* src, const VSFrameInfo* fi); /* :111 */
VS_API void vsFrameFillFromBuffer(VSFrame* frame, uint8_t* img, const VSFrameInfo* fi); /* :117 */
VS_API void vsFrameFree(VSFrame* frame);                               /* :120 */

/* ---- growable pointer vector: src/vsvector.h:35-222 ----------------------- */
typedef struct vsvector_ VSVector;
struct vsvector_ {
  void** data;
  int buffersize;
  int nelems;
};
#define VS_VECTOR_MAX_SIZE ((int)(2147483647 / sizeof(void*)))

VS_API int vs_vector_init(VSVector* V, int buffersize);                /* src/vsvector.h:54 */
VS_API int vs_vector_fini(VSVector* V);                                /* :67 */
VS_API int vs_vector_del(VSVector* V);                                 /* :79 */
VS_API int vs_vector_zero(VSVector* V);                                /* :86 */
VS_API int vs_vector_size(const VSVector* V);                          /* :99 */
VS_API int vs_vector_append(VSVector* V, void* data);                  /* :118 */
VS_API int vs_vector_append_dup(VSVector* V, void* data, int data_size); /* :124 */
VS_API int vs_vector_set(VSVector* V, int pos, void* data, void** old); /* :152 */
VS_API int vs_vector_set_dup(VSVector* V, int pos, void* data, int data_size,
                             void** old);                              /* :158 */
VS_API void* vs_vector_get(const VSVector* V, int pos);                /* :172 */
VS_API VSVector vs_vector_filter(const VSVector* V, short (*pred)(void*, void*),
                                 void* param);                         /* :179 */
VS_API VSVector vs_vector_concat(const VSVector* V1, const VSVector* V2); /* :185 */

typedef struct vsarray_ VSArray;
struct vsarray_ {
  double* dat;
  int len;
};
VS_API VSArray vs_array(double vals[], int len);                       /* :198 */
VS_API VSArray vs_array_new(int len);                                  /* :201 */
VS_API VSArray* vs_array_plus(VSArray* c, VSArray a, VSArray b);       /* :204 */
VS_API VSArray* vs_array_scale(VSArray* c, VSArray a, double f);       /* :207 */
VS_API VSArray vs_array_copy(VSArray a);                               /* :210 */
VS_API void vs_array_zero(VSArray* a);                                 /* :213 */
VS_API void vs_array_swap(VSArray* a, VSArray* b);                     /* :216 */
VS_API void vs_array_free(VSArray a);                                  /* :219 */
VS_API void vs_array_print(VSArray a, FILE* f);                        /* :222 */

/* ---- result types: src/transformtype.h:38-71 ------------------------------ */
typedef struct _transform {
  double x;
  double y;
  double alpha;
  double zoom;
  double barrel;
  double rshutter;
  int extra;
} VSTransform;

typedef struct _field {
  int16_t x;    /* centre */
  int16_t y;
  int16_t size; /* edge length in pixels */
} Field;

typedef struct _vec {
  int16_t x;
  int16_t y;
} Vec;

typedef struct _localmotion {
  Vec v;           /* displacement of the field centre, previous -> current */
  Field f;         /* the measurement field */
  double contrast; /* Michelson contrast of the field */
  double match;    /* SAD of the best shift per pixel */
} LocalMotion;

typedef VSVector LocalMotions;

#define LMGet(localmotions, index) ((LocalMotion*)vs_vector_get(localmotions, index))

/* ---- transform helpers used by the detect pass:
        src/transformtype_operations.h:44-173, src/localmotion2transform.h --- */
typedef struct _preparedtransform {
  const VSTransform* t;
  double zcos_a;
  double zsin_a;
  double c_x;
  double c_y;
  double f;
  double z;
  double r[9];
} PreparedTransform;                                                   /* :56-68 */

VS_API VSTransform null_transform(void);                               /* :44 */
VS_API VSTransform new_transform(double x, double y, double alpha, double zoom,
                                 double barrel, double rshutter, int extra); /* :45 */
VS_API VSTransform add_transforms(const VSTransform* t1, const VSTransform* t2); /* :47 */
VS_API VSTransform sub_transforms(const VSTransform* t1, const VSTransform* t2); /* :49 */
VS_API VSTransform mult_transform(const VSTransform* t1, double f);    /* :50 */
VS_API void storeVSTransform(FILE* f, const VSTransform* t);           /* :53 */
VS_API PreparedTransform prepare_transform(const VSTransform* t, const VSFrameInfo* fi); /* :97 */
VS_API Vec transform_vec(const PreparedTransform* t, const Vec* v);    /* :103 */
VS_API void transform_vec_double(double* x, double* y, const PreparedTransform* t,
                                 const Vec* v);                        /* :104 */
VS_API Vec sub_vec(Vec v1, Vec v2);                                    /* :107 */
VS_API Vec add_vec(Vec v1, Vec v2);                                    /* :109 */
VS_API Vec field_to_vec(Field f);                                      /* :110 */
VS_API int cmp_double(const void* t1, const void* t2);                 /* :119 */
VS_API int cmp_int(const void* t1, const void* t2);                    /* :121 */
VS_API double cleanmean(double* ds, int len, double* minimum, double* maximum); /* :140 */
VS_API LocalMotion null_localmotion(void);                             /* :160 */
VS_API int* localmotions_getx(const LocalMotions* localmotions);       /* :162 */
VS_API int* localmotions_gety(const LocalMotions* localmotions);       /* :164 */
VS_API LocalMotion sub_localmotion(const LocalMotion* lm1, const LocalMotion* lm2); /* :166 */
VS_API LocalMotion cleanmean_localmotions(const LocalMotions* localmotions); /* :171 */
VS_API VSArray localmotionsGetMatch(const LocalMotions* localmotions); /* :173 */
/* src/localmotion2transform.h: the simple coarse-motion model the detect
   pass uses to centre the fine search */
VS_API double vsCalcAngle(const LocalMotion* lm, int center_x, int center_y);
VS_API VSTransform vsSimpleMotionsToTransform(VSFrameInfo fi, const char* modName,
                                              const LocalMotions* motions);

/* ---- detect: src/motiondetect.h:42-147 ----------------------------------- */
#define ASCII_SERIALIZATION_MODE 1
#define BINARY_SERIALIZATION_MODE 2

typedef struct _vsmotiondetectconfig {
  int shakiness;            /* 1..10, only enters through the accuracy clamp */
  int accuracy;             /* 1..15: share of measurement fields used */
  int stepSize;             /* lattice step of the coarse search */
  int algo;                 /* unused */
  int virtualTripod;        /* >0: compare against frame virtualTripod-1 */
  int show;                 /* 1,2: draw fields and shifts into the frame */
  double contrastThreshold; /* fields of lower contrast are dropped */
  const char* modName;      /* tag for vs_log */
  int numThreads;           /* host threads (the GPU path ignores it) */
} VSMotionDetectConfig;

typedef struct _vsmotiondetectfields {
  int maxShift;
  int stepSize;
  int fieldNum;
  int maxFields;
  double contrastThreshold;
  int fieldSize;
  int fieldRows;
  Field* fields;
  short useOffset;
  VSTransform offset;
} VSMotionDetectFields;

/* Caller-allocated; its layout is ABI.  The GPU path keeps its device state
   in a table keyed by the address of this struct; the frame members curr,
   currtmp and prev are left null (they are internal in the reference too). */
typedef struct _vsmotiondetect {
  VSFrameInfo fi;
  VSMotionDetectConfig conf;
  VSMotionDetectFields fieldscoarse;
  VSMotionDetectFields fieldsfine;
  VSFrame curr;
  VSFrame currorig;
  VSFrame currtmp;
  VSFrame prev;
  short hasSeenOneFrame;
  int initialized;
  int serializationMode;
  int frameNum;
} VSMotionDetect;

VS_API VSMotionDetectConfig vsMotionDetectGetDefaultConfig(const char* modName); /* src/motiondetect.h:121 */
VS_API int vsMotionDetectInit(VSMotionDetect* md, const VSMotionDetectConfig* conf,
                              const VSFrameInfo* fi);                  /* :127 */
VS_API int vsMotionDetection(VSMotionDetect* md, LocalMotions* motions, VSFrame* frame); /* :136 */
VS_API void vsMotionDetectionCleanup(VSMotionDetect* md);              /* :141 */
VS_API void vsMotionDetectGetConfig(VSMotionDetectConfig* conf, const VSMotionDetect* md); /* :144 */
VS_API const VSFrameInfo* vsMotionDetectGetFrameInfo(const VSMotionDetect* md); /* :147 */

/* ---- .trf serialization: src/serialize.h:58-98 ---------------------------- */
#define LIBVIDSTAB_FILE_FORMAT_VERSION 1
typedef VSVector VSManyLocalMotions;
#define VSMLMGet(manylocalmotions, index) \
  ((LocalMotions*)vs_vector_get(manylocalmotions, index))

VS_API int vsGuessSerializationMode(FILE* f);                          /* src/serialize.h:65 */
VS_API int vsStoreLocalmotions(FILE* f, const LocalMotions* lms, const int serializationMode); /* :68 */
VS_API LocalMotions vsRestoreLocalmotions(FILE* f, const int serializationMode); /* :71 */
VS_API int vsPrepareFile(const VSMotionDetect* td, FILE* f);           /* :75 */
VS_API int vsWriteToFile(const VSMotionDetect* td, FILE* f, const LocalMotions* lms); /* :78 */
VS_API int vsReadFileVersion(FILE* f, const int serializationMode);    /* :81 */
VS_API int vsReadFromFile(FILE* f, LocalMotions* lms, const int serializationMode); /* :87 */
VS_API int vsReadLocalMotionsFile(FILE* f, VSManyLocalMotions* lms);   /* :98 */

/* ---- second pass: local motions -> one global transform per frame --------
   The transform pass's configuration, read through the caller's pointer, with
   the reference's member order and sizes (src/transform.h:60-66, :88-160,
   src/lensmap.h:52-110).  Only fiSrc and conf are read here; the remaining
   members are declared so that offsets and size agree. */
typedef enum { VS_Zero, VS_Linear, VS_BiLinear, VS_BiCubic, VS_NBInterPolTypes } VSInterpolType;
typedef enum { VSKeepBorder = 0, VSCropBorder } VSBorderType;
typedef enum { VSOptimalL1 = 0, VSGaussian, VSAvg } VSCamPathAlgo;
typedef enum { VSLensCorrectOff = 0, VSLensCorrectWobble, VSLensCorrectFull } VSLensCorrectMode;
typedef void (*vsInterpolateFun)(uint8_t* rv, int32_t x, int32_t y, const uint8_t* img,
                                 int linesize, int width, int height, uint8_t def);

typedef struct _VSTransformConfig {
  int relative;
  int smoothing;
  VSBorderType crop;
  int invert;
  double zoom;
  int optZoom;
  double zoomSpeed;
  VSInterpolType interpolType;
  int maxShift;
  double maxAngle;
  const char* modName;
  int verbose;
  int simpleMotionCalculation;  /* 1: vsSimpleMotionsToTransform per frame */
  int storeTransforms;          /* write global_motions.trf */
  int smoothZoom;               /* 0: the fitted zoom is dropped */
  VSCamPathAlgo camPathAlgo;
  int estimateLensDistortion;   /* the lens estimate is not supported: must be 0
                                   unless simpleMotionCalculation is set */
  VSLensCorrectMode lensCorrection;
  double lensK;
  double fov;                   /* > 0: rotational model, degrees across the width */
} VSTransformConfig;

typedef struct _vslensplanemap {
  int active;
  VSLensCorrectMode mode;
  double k, cdx, cdy, csx, csy, tMaxU, tMaxD, tDomD, invRho2, f;
  int sxShift, syShift;
  int32_t idxScaleU, idxScaleD;
  int32_t* gU;
  int32_t* gD;
} VSLensPlaneMap;

typedef struct _VSTransformData {
  VSFrameInfo fiSrc;
  VSFrameInfo fiDest;
  VSFrame src;
  VSFrame destbuf;
  VSFrame dest;
  short srcMalloced;
  vsInterpolateFun interpolate;
  VSTransformConfig conf;
  VSLensCorrectMode lensMode;
  int lensActive;
  double lensK;
  double lensMapK;
  VSLensPlaneMap lensMaps[3];
  int initialized;
} VSTransformData;

typedef struct _vstransformations {  /* src/transform.h:44-49 */
  VSTransform* ts;
  int current;
  int len;
  short warned_end;
} VSTransformations;

/* Fits one transform per frame of `motions` (src/localmotion2transform.c:
   40-121): the similarity model (or the rotational one when conf.fov > 0) by
   the reference's masked gradient descent, every frame on the GPU at once; or
   vsSimpleMotionsToTransform per frame when conf.simpleMotionCalculation is
   set.  trans->ts is allocated with vs_malloc and trans->len set.  With
   conf.storeTransforms the per-frame lines of global_motions.trf are written
   as the reference writes them.  VS_ERROR (and a log line) when
   conf.estimateLensDistortion is set without simpleMotionCalculation, or on a
   device failure. */
VS_API int vsLocalmotions2Transforms(VSTransformData* td, const VSManyLocalMotions* motions,
                                     VSTransformations* trans);  /* src/localmotion2transform.h:38 */
/* One frame of the above (src/localmotion2transform.c:220-284); f, when not
   NULL, receives the frame's global_motions.trf line. */
VS_API VSTransform vsMotionsToTransform(VSTransformData* td, const LocalMotions* motions,
                                        FILE* f);               /* src/localmotion2transform.h:65 */

#ifdef __cplusplus
}
#endif

#include "vidstab_b200_ext.h"

#endif /* VIDSTAB_B200_H */
