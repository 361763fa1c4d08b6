/*
 * format.h -- JPEG reader, marker parser and decode driver of libcudajpeg.
 *
 * Drop-in for the reference's include/format.h (jndean/CUDAjpeg): the same
 * entry points, error codes and reader fields that callers touch, with C
 * linkage so the reference's src/main.cu (or any C/C++/FFI caller) links
 * against libcudajpeg.so unchanged.
 *
 *   reference                          here
 *   newJPGReader   format.h:106        newJPGReader   (allocates host state only)
 *   delJPGReader   format.h:105        delJPGReader
 *   openJPG        format.h:108        openJPG        (whole decode on the GPU)
 *   writeJPG       format.h:109        writeJPG       (PPM / PGM)
 *   printError     format.h:110        printError
 *   read16, skipBlock, decodeSOF/DHT/DQT/DRI  format.h:105-115  same names
 *
 * openJPG returns 0 or one of the error codes below and leaves the output in
 * reader->pixels (interleaved RGB, width*height*3) for colour images or in
 * reader->channels[0].pixels.mem (width*height) for greyscale, as in the
 * reference (src/format.cu:218-229).
 */
#ifndef FORMAT_H
#define FORMAT_H

#include <stddef.h>
#include <stdint.h>
#include <time.h>

/* Error codes: include/format.h:7-14 of the reference */
#define NO_ERROR 0
#define SYNTAX_ERROR 1
#define UNSUPPORTED_ERROR 2
#define OOM_ERROR 3
#define CUDA_MEM_ERROR 4
#define FILE_ERROR 5
#define CUDA_KERNEL_LAUNCH_ERROR 6
#define PROGRAMMER_ERROR -1

/* Memory options for ensureMemSize (reference format.h:16-19) */
#define USE_MALLOC 0
#define USE_CALLOC 1
#define USE_CUDA_MALLOC 2

/* Records the error and where it was raised, then returns (format.h:22-27). */
#define THROW(e)                          \
  do {                                    \
    jpg->error = (e);                     \
    jpg->error_line = __LINE__;           \
    jpg->error_file = (char *)__FILE__;   \
    jpg->error_func = (char *)__func__;   \
    return;                               \
  } while (0)

#ifdef __cplusplus
extern "C" {
#endif

typedef struct _DhtVlc {
  unsigned char tuple, num_bits;
} DhtVlc;

typedef struct _ManagedUCharMem {
  unsigned char *mem;
  unsigned int size, max_size;
} ManagedUCharMem;

typedef struct _ManagedShortMem {
  short *mem;
  unsigned int size, max_size;
} ManagedShortMem;

typedef struct _ManagedIntMem {
  int *mem;
  unsigned int size, max_size;
} ManagedIntMem;

typedef struct _ColourChannel {
  int id;
  int dq_id, ac_id, dc_id;
  int width, height;                 /* component size in pixels */
  int samples_x, samples_y, stride;  /* sampling factors; padded plane stride */
  int block_stride;                  /* padded plane rows (whole MCUs) */
  int num_blocks;                    /* 8x8 blocks of this component */
  int dc_cumulative_val;             /* kept for layout compatibility */
  ManagedIntMem working_space;       /* int32 dequantised coefficients, filled
                                        on the host only when the reader flag
                                        CJ_READER_HOST_COEFFICIENTS is set */
  ManagedUCharMem pixels;            /* channel 0: greyscale output */
} ColourChannel;

struct CJReaderDevice; /* opaque: stream, device buffers, pinned staging */

typedef struct _JPGReader {
  /* File buffer pointers: buf owns the file bytes (pinned host memory);
     pos / end walk the marker segments. */
  unsigned char *buf, *pos, *end;
  /* Image properties */
  unsigned short width, height;
  unsigned short num_blocks_x, num_blocks_y; /* MCUs across / down */
  unsigned short block_size_x, block_size_y; /* MCU size in pixels */
  unsigned char num_channels;
  int restart_interval;
  ColourChannel channels[3];
  /* Output */
  unsigned char *pixels; /* RGB, width*height*3, pinned host memory */
  int max_pixels_size;
  unsigned char dq_tables[4][64];
  ManagedUCharMem file_buf;
  /* Timing: accumulated device time of the last decode, in clock() ticks
     (main.cu:47 sums it as DEBUG_TIME) */
  clock_t time;
  /* Errors (set through THROW) */
  int error, error_line;
  char *error_file, *error_func;
  /* libcudajpeg additions */
  int flags;                     /* CJ_READER_* */
  int scan_seen;                 /* an SOS was decoded in this file */
  int huff_defined;              /* bit i: Huffman slot i defined */
  struct CJReaderDevice *dev;
} JPGReader;

/* reader->flags */
#define CJ_READER_HOST_COEFFICIENTS 1 /* also copy coefficients to working_space */

unsigned short read16(const unsigned char *pos);
void delJPGReader(JPGReader *reader);
JPGReader *newJPGReader(void);
int openJPG(JPGReader *reader, const char *filename);
void writeJPG(JPGReader *jpg, const char *filename);
void printError(JPGReader *reader);
void skipBlock(JPGReader *jpg);
void decodeSOF(JPGReader *jpg);
void decodeDHT(JPGReader *jpg);
void decodeDQT(JPGReader *jpg);
void decodeDRI(JPGReader *jpg);

/* libcudajpeg addition: decode a JPEG already in host memory (same result
   and error codes as openJPG on a file with these bytes). */
int openJPGMem(JPGReader *reader, const unsigned char *data, size_t size);

#ifdef __cplusplus
}
#endif

/* Natural-order index of each zig-zag position (reference format.h:117-120) */
static const char deZigZag[64] = {
    0,  1,  8,  16, 9,  2,  3,  10, 17, 24, 32, 25, 18, 11, 4,  5,  12, 19, 26, 33, 40, 48,
    41, 34, 27, 20, 13, 6,  7,  14, 21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15,
    23, 30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53, 60, 61, 54, 47, 55, 62, 63};

#endif /* FORMAT_H */
