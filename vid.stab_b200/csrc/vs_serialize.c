/*
 * vs_serialize.c -- the .trf file the detect pass writes (format of
 * src/serialize.c:168-409 of the reference, byte for byte, and its readers
 * :411-561).  Little-endian hosts only (x86-64 / aarch64 little endian),
 * which is what the format stores.
 *
 *   binary:  "TRF" <version as decimal text> int32 accuracy, shakiness,
 *            stepsize, double mincontrast; then per frame int32 frameNum,
 *            int32 n, n x (int16 v.x v.y f.x f.y f.size, double contrast,
 *            double match)
 *   text:    "VID.STAB 1" header with '#' comment lines, then per frame
 *            "Frame <n> (List <k> [(LM vx vy fx fy size contrast match),...])"
 */
#include <string.h>

#include "vidstab_b200.h"

#if defined(__BYTE_ORDER__) && __BYTE_ORDER__ == __ORDER_BIG_ENDIAN__
#error "the .trf binary format is little endian; big-endian hosts are not supported"
#endif

static const char* kTag = "vid.stab - serialization";

/* per-frame and per-file sanity limits of the reader (src/serialize.c:93,101) */
#define TRF_MAX_MOTIONS (1 << 20)
#define TRF_MAX_FRAMES (1 << 22)

static int put16(FILE* f, int16_t v) { return (int)fwrite(&v, sizeof(v), 1, f); }
static int put32(FILE* f, int32_t v) { return (int)fwrite(&v, sizeof(v), 1, f); }
static int putd(FILE* f, double v) { return (int)fwrite(&v, sizeof(v), 1, f); }
static int get16(FILE* f, int16_t* v) { return (int)fread(v, sizeof(*v), 1, f); }
static int get32(FILE* f, int32_t* v) { return (int)fread(v, sizeof(*v), 1, f); }
static int getd(FILE* f, double* v) { return (int)fread(v, sizeof(*v), 1, f); }

static void binary_read_failed(FILE* f, const char* what) {
  if (f && feof(f))
    vs_log_error(kTag,
                 "Cannot parse %s: unexpected end of file. The transform file is "
                 "truncated or corrupt; write and read it through a handle opened in "
                 "binary mode (\"wb\" / \"rb\").\n",
                 what);
  else
    vs_log_error(kTag, "Cannot parse %s: read error or malformed record!\n", what);
}

static int put_lm_binary(FILE* f, const LocalMotion* lm) {
  return put16(f, lm->v.x) > 0 && put16(f, lm->v.y) > 0 && put16(f, lm->f.x) > 0 &&
         put16(f, lm->f.y) > 0 && put16(f, lm->f.size) > 0 && putd(f, lm->contrast) > 0 &&
         putd(f, lm->match) > 0;
}

static int get_lm_binary(FILE* f, LocalMotion* lm) {
  return get16(f, &lm->v.x) > 0 && get16(f, &lm->v.y) > 0 && get16(f, &lm->f.x) > 0 &&
         get16(f, &lm->f.y) > 0 && get16(f, &lm->f.size) > 0 && getd(f, &lm->contrast) > 0 &&
         getd(f, &lm->match) > 0;
}

static int put_lm_text(FILE* f, const LocalMotion* lm) {
  return fprintf(f, "(LM %hi %hi %hi %hi %hi %lf %lf)", lm->v.x, lm->v.y, lm->f.x, lm->f.y,
                 lm->f.size, lm->contrast, lm->match);
}

static LocalMotion get_lm_text(FILE* f) {
  LocalMotion lm;
  int c;
  if (fscanf(f, "(LM %hi %hi %hi %hi %hi %lf %lf", &lm.v.x, &lm.v.y, &lm.f.x, &lm.f.y,
             &lm.f.size, &lm.contrast, &lm.match) != 7) {
    vs_log_error(kTag, "Cannot parse localmotion!\n");
    return null_localmotion();
  }
  while ((c = fgetc(f)) && c != ')' && c != EOF) {
  }
  if (c == EOF) {
    vs_log_error(kTag, "Cannot parse localmotion missing ')'!\n");
    return null_localmotion();
  }
  return lm;
}

int vsStoreLocalmotions(FILE* f, const LocalMotions* lms, const int mode) {
  int n = vs_vector_size(lms);
  if (mode == BINARY_SERIALIZATION_MODE) {
    if (put32(f, n) <= 0) return 0;
    for (int i = 0; i < n; i++)
      if (!put_lm_binary(f, LMGet(lms, i))) return 0;
    return 1;
  }
  fprintf(f, "List %i [", n);
  for (int i = 0; i < n; i++) {
    if (i > 0) fprintf(f, ",");
    if (put_lm_text(f, LMGet(lms, i)) <= 0) return 0;
  }
  fprintf(f, "]");
  return 1;
}

LocalMotions vsRestoreLocalmotions(FILE* f, const int mode) {
  LocalMotions lms;
  int32_t len;
  int c;
  vs_vector_init(&lms, 0);
  if (mode == BINARY_SERIALIZATION_MODE) {
    if (get32(f, &len) <= 0) {
      binary_read_failed(f, "localmotions list");
      return lms;
    }
    if (len < 0 || len > TRF_MAX_MOTIONS) {
      vs_log_error(kTag, "Implausible number of localmotions (%i): the transform file is corrupt!\n",
                   len);
      return lms;
    }
    if (len > 0) {
      vs_vector_init(&lms, len);
      for (int i = 0; i < len; i++) {
        LocalMotion lm;
        if (!get_lm_binary(f, &lm)) {
          binary_read_failed(f, "localmotion");
          break;
        }
        vs_vector_append_dup(&lms, &lm, sizeof(LocalMotion));
      }
    }
    if (len != vs_vector_size(&lms))
      vs_log_error(kTag, "Cannot parse the given number of localmotions (got %i of %i)!\n",
                   vs_vector_size(&lms), len);
    return lms;
  }
  int tlen;
  if (fscanf(f, "List %i [", &tlen) != 1) {
    vs_log_error(kTag, "Cannot parse localmotions list expect 'List len ['!\n");
    return lms;
  }
  if (tlen > 0) {
    vs_vector_init(&lms, tlen);
    for (int i = 0; i < tlen; i++) {
      if (i > 0)
        while ((c = fgetc(f)) && c != ',' && c != EOF) {
        }
      LocalMotion lm = get_lm_text(f);
      vs_vector_append_dup(&lms, &lm, sizeof(LocalMotion));
    }
  }
  if (tlen != vs_vector_size(&lms)) {
    vs_log_error(kTag, "Cannot parse the given number of localmotions!\n");
    return lms;
  }
  while ((c = fgetc(f)) && c != ']' && c != EOF) {
  }
  if (c == EOF) vs_log_error(kTag, "Cannot parse localmotions list missing ']'!\n");
  return lms;
}

int vsPrepareFile(const VSMotionDetect* md, FILE* f) {
  if (!f) return VS_ERROR;
  if (md->serializationMode == BINARY_SERIALIZATION_MODE) {
    fprintf(f, "TRF%hhu", (unsigned char)LIBVIDSTAB_FILE_FORMAT_VERSION);
    put32(f, md->conf.accuracy);
    put32(f, md->conf.shakiness);
    put32(f, md->conf.stepSize);
    putd(f, md->conf.contrastThreshold);
    return VS_OK;
  }
  fprintf(f, "VID.STAB %i\n", LIBVIDSTAB_FILE_FORMAT_VERSION);
  fprintf(f, "#      accuracy = %d\n", md->conf.accuracy);
  fprintf(f, "#     shakiness = %d\n", md->conf.shakiness);
  fprintf(f, "#      stepsize = %d\n", md->conf.stepSize);
  fprintf(f, "#   mincontrast = %f\n", md->conf.contrastThreshold);
  return VS_OK;
}

int vsWriteToFile(const VSMotionDetect* md, FILE* f, const LocalMotions* lms) {
  if (!f || !lms) return VS_ERROR;
  if (md->serializationMode == BINARY_SERIALIZATION_MODE) {
    if (put32(f, md->frameNum) <= 0) return VS_ERROR;
    if (vsStoreLocalmotions(f, lms, BINARY_SERIALIZATION_MODE) <= 0) return VS_ERROR;
    return VS_OK;
  }
  if (fprintf(f, "Frame %i (", md->frameNum) > 0 &&
      vsStoreLocalmotions(f, lms, ASCII_SERIALIZATION_MODE) > 0 && fprintf(f, ")\n"))
    return VS_OK;
  return VS_ERROR;
}

int vsGuessSerializationMode(FILE* f) {
  int mode = ASCII_SERIALIZATION_MODE;
  long pos = ftell(f);
  if (fgetc(f) == 'T' && fgetc(f) == 'R' && fgetc(f) == 'F') mode = BINARY_SERIALIZATION_MODE;
  fseek(f, pos, SEEK_SET);
  return mode;
}

int vsReadFileVersion(FILE* f, const int mode) {
  if (!f) return VS_ERROR;
  if (mode == BINARY_SERIALIZATION_MODE) {
    unsigned char version;
    int32_t a, s, st;
    double mc;
    if (fscanf(f, "TRF%hhu", &version) != LIBVIDSTAB_FILE_FORMAT_VERSION) return VS_ERROR;
    if (get32(f, &a) <= 0 || get32(f, &s) <= 0 || get32(f, &st) <= 0 || getd(f, &mc) <= 0)
      return VS_ERROR;
    return version;
  }
  int version;
  if (fscanf(f, "VID.STAB %i\n", &version) != LIBVIDSTAB_FILE_FORMAT_VERSION) return VS_ERROR;
  return version;
}

int vsReadFromFile(FILE* f, LocalMotions* lms, const int mode) {
  if (mode == BINARY_SERIALIZATION_MODE) {
    int32_t frameNum;
    if (get32(f, &frameNum) <= 0) return VS_ERROR;
    *lms = vsRestoreLocalmotions(f, BINARY_SERIALIZATION_MODE);
    return frameNum;
  }
  for (;;) {
    int c = fgetc(f);
    if (c == 'F') {
      int num;
      if (fscanf(f, "rame %i (", &num) != 1) {
        vs_log_error(kTag, "cannot read file, expect 'Frame num (...'");
        return VS_ERROR;
      }
      *lms = vsRestoreLocalmotions(f, ASCII_SERIALIZATION_MODE);
      if (fscanf(f, ")\n") < 0) {
        vs_log_error(kTag, "cannot read file, expect '...)'");
        return VS_ERROR;
      }
      return num;
    } else if (c == '#') {
      char line[1024];
      if (fgets(line, sizeof(line), f) == 0) return VS_ERROR;
    } else if (c == '\n' || c == '\r' || c == ' ' || c == '\t') {
      /* whitespace between records, CRLF line ends included */
    } else if (c == EOF) {
      return VS_ERROR;
    } else {
      vs_log_error(kTag, "cannot read frame local motions from file, got %c (%i)", c, c);
      return VS_ERROR;
    }
  }
}

static void free_many(VSManyLocalMotions* m) {
  for (int i = 0; i < vs_vector_size(m); i++) {
    LocalMotions* l = (LocalMotions*)vs_vector_get(m, i);
    if (l) vs_vector_del(l);
  }
  vs_vector_del(m);
}

int vsReadLocalMotionsFile(FILE* f, VSManyLocalMotions* mlms) {
  int mode = vsGuessSerializationMode(f);
  int version = vsReadFileVersion(f, mode);
  if (version < 1) return VS_ERROR;
  if (version > 1) {
    vs_log_error(kTag, "Version of VID.STAB file too large: got %i, expect <= 1", version);
    return VS_ERROR;
  }
  if (vs_vector_init(mlms, 1024) != VS_OK) return VS_ERROR;
  int index, last = 0;
  LocalMotions lms;
  while ((index = vsReadFromFile(f, &lms, mode)) != VS_ERROR) {
    if (index > last + 1)
      vs_log_info(kTag, "VID.STAB file: index of frames is not continuous %i -< %i", last, index);
    if (index < 1 || index > TRF_MAX_FRAMES) {
      vs_log_info(kTag, "VID.STAB file: implausible frame number (%i), expect 1..%i", index,
                  TRF_MAX_FRAMES);
      vs_vector_del(&lms);
    } else {
      void* old = 0;
      if (vs_vector_set_dup(mlms, index - 1, &lms, sizeof(LocalMotions), &old) != VS_OK) {
        vs_log_error(kTag, "VID.STAB file: cannot store the localmotions of frame %i", index);
        vs_vector_del(&lms);
        free_many(mlms);
        return VS_ERROR;
      }
      if (old) {
        vs_vector_del((LocalMotions*)old);
        vs_free(old);
      }
    }
    last = index;
  }
  return VS_OK;
}
