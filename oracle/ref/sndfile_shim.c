/*
 * Test infrastructure for the oracle: a WAV-only stand-in for the six libsndfile
 * entry points the reference loads with dlopen (src/io/audio.cpp:62-84), so the
 * reference planner can decode sample banks in a container without libsndfile.
 *
 * Supported: RIFF/WAVE with PCM 16/24/32-bit integer or 32-bit float data, mono or
 * stereo, read mode only.  Integers are scaled by 2^-(bits-1), which is exact in
 * float32 and matches libsndfile's normalised sf_readf_float for these formats.
 * SFC_GET_INSTRUMENT (0x10d0) reports forward loops from a `smpl` chunk with the
 * end made exclusive (end + 1).  Write mode (FLAC output) is refused.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int64_t frames;
    int samplerate, channels, format, sections, seekable;
} SF_INFO;

typedef struct {
    int gain;
    char basenote, detune, velocity_lo, velocity_hi, key_lo, key_hi;
    int loop_count;
    struct { int mode; unsigned start, end, count; } loops[16];
} SF_INSTRUMENT;

typedef struct {
    unsigned char* data;     /* whole file */
    size_t size;
    const unsigned char* pcm;
    int64_t frames, position;
    int channels, bits, is_float, rate;
    int has_loop;
    unsigned loop_start, loop_end;
} Shim;

static uint32_t le32(const unsigned char* p) { return p[0] | (p[1] << 8) | (p[2] << 16) | ((uint32_t)p[3] << 24); }
static uint16_t le16(const unsigned char* p) { return (uint16_t)(p[0] | (p[1] << 8)); }

void* sf_open(const char* path, int mode, SF_INFO* info)
{
    if (mode != 0x10)
        return NULL;
    FILE* f = fopen(path, "rb");
    if (!f)
        return NULL;
    fseek(f, 0, SEEK_END);
    long size = ftell(f);
    fseek(f, 0, SEEK_SET);
    if (size < 12) { fclose(f); return NULL; }
    Shim* s = calloc(1, sizeof *s);
    s->data = malloc((size_t)size);
    s->size = (size_t)size;
    if (fread(s->data, 1, (size_t)size, f) != (size_t)size) { fclose(f); free(s->data); free(s); return NULL; }
    fclose(f);
    if (memcmp(s->data, "RIFF", 4) || memcmp(s->data + 8, "WAVE", 4)) goto fail;
    size_t pos = 12;
    int format = 0;
    while (pos + 8 <= s->size) {
        const unsigned char* chunk = s->data + pos;
        uint32_t length = le32(chunk + 4);
        if (pos + 8 + length > s->size) length = (uint32_t)(s->size - pos - 8);
        if (!memcmp(chunk, "fmt ", 4) && length >= 16) {
            format = le16(chunk + 8);
            s->channels = le16(chunk + 10);
            s->rate = (int)le32(chunk + 12);
            s->bits = le16(chunk + 22);
            if (format == 0xFFFE && length >= 40) format = le16(chunk + 8 + 24);
        } else if (!memcmp(chunk, "data", 4)) {
            s->pcm = chunk + 8;
            s->frames = s->channels && s->bits ? length / (s->channels * (s->bits / 8)) : 0;
        } else if (!memcmp(chunk, "smpl", 4) && length >= 36 + 24) {
            uint32_t loops = le32(chunk + 8 + 28);
            if (loops > 0 && le32(chunk + 8 + 36 + 4) == 0) {
                s->has_loop = 1;
                s->loop_start = le32(chunk + 8 + 36 + 8);
                s->loop_end = le32(chunk + 8 + 36 + 12) + 1;
            }
        }
        pos += 8 + length + (length & 1);
    }
    if (!s->pcm || (format != 1 && format != 3)) goto fail;
    s->is_float = format == 3;
    if (s->is_float ? s->bits != 32 : (s->bits != 16 && s->bits != 24 && s->bits != 32)) goto fail;
    info->frames = s->frames;
    info->samplerate = s->rate;
    info->channels = s->channels;
    info->format = 0x010000 | (s->is_float ? 0x0006 : s->bits == 16 ? 0x0002 : s->bits == 24 ? 0x0003 : 0x0004);
    info->sections = 1;
    info->seekable = 1;
    return s;
fail:
    free(s->data);
    free(s);
    return NULL;
}

int sf_close(void* handle)
{
    Shim* s = handle;
    if (s) { free(s->data); free(s); }
    return 0;
}

int64_t sf_readf_float(void* handle, float* out, int64_t frames)
{
    Shim* s = handle;
    int64_t count = s->frames - s->position;
    if (frames < count) count = frames;
    const int width = s->bits / 8;
    const unsigned char* p = s->pcm + (size_t)s->position * s->channels * width;
    for (int64_t i = 0; i < count * s->channels; ++i, p += width) {
        float value;
        if (s->is_float) {
            memcpy(&value, p, 4);
        } else if (width == 2) {
            value = (float)(int16_t)le16(p) * (1.0f / 32768.0f);
        } else if (width == 3) {
            int32_t v = (int32_t)((uint32_t)p[0] << 8 | (uint32_t)p[1] << 16 | (uint32_t)p[2] << 24) >> 8;
            value = (float)v * (1.0f / 8388608.0f);
        } else {
            value = (float)((double)(int32_t)le32(p) * (1.0 / 2147483648.0));
        }
        out[i] = value;
    }
    s->position += count;
    return count;
}

int sf_command(void* handle, int command, void* data, int size)
{
    Shim* s = handle;
    if (command == 0x10d0 && s && s->has_loop && size >= (int)sizeof(SF_INSTRUMENT)) {
        SF_INSTRUMENT* inst = data;
        memset(inst, 0, sizeof *inst);
        inst->loop_count = 1;
        inst->loops[0].mode = 801;
        inst->loops[0].start = s->loop_start;
        inst->loops[0].end = s->loop_end;
        return 1;
    }
    return 0;
}

int64_t sf_writef_short(void* handle, const int16_t* data, int64_t frames)
{
    (void)handle; (void)data; (void)frames;
    return 0;
}

int sf_error(void* handle)
{
    (void)handle;
    return 0;
}
