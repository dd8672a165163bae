/*
 * claysampler_b200 host library — the C++17 planner and file I/O in front of the
 * GPU renderer (include/claysampler_b200.h).
 *
 * cs_host_plan turns one job (SFZ instrument + Standard MIDI File) into a plan
 * image exactly as the reference CLI's planBatch does (src/main.cpp:298-361, with
 * src/sfz/instrument.cpp, src/io/midi.cpp and src/render/plan.cpp), decoding the
 * samples that trigger into the host's shared float32 bank.  All entry points
 * return 0 on success; cs_host_last_error() gives the message otherwise.
 */
#ifndef CLAYSAMPLER_HOST_H
#define CLAYSAMPLER_HOST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct cs_host cs_host;

int cs_host_create(cs_host** out);
void cs_host_destroy(cs_host* host);

/* tail: 0 natural, 1 orig, 2 custom (--tail-policy).  max_audio / tail_max are
 * seconds, negative when not given (--max-audio-seconds, --tail-max-seconds);
 * tail_fade_ms < 0 means the default 100 ms (--tail-fade-ms).  `quality` keeps
 * the MIDI onsets for the quality gate; `group` is the volume-group id (0 = none).
 * On success *image holds the plan image (claysampler_b200/csrc/plan_blob.hpp
 * layout, free with cs_host_free) whose spans index into the host's bank. */
int cs_host_plan(cs_host* host, const char* sfz, const char* midi, int rate, int tail, double max_audio,
                 double tail_max, int tail_fade_ms, int quality, int group_volume, uint64_t group,
                 void** image, size_t* size);
void cs_host_free(void* pointer);

/* Loads one SFZ preset with a private bank and reports its region count: the
 * reference CLI's --check-sfz (src/main.cpp:264-287). */
int cs_host_check_sfz(const char* sfz, int* regions);

/* The shared decoded bank (AudioBank::pcm, src/io/audio.h:32); valid until the
 * next cs_host_plan or cs_host_release_bank. */
int cs_host_bank(cs_host* host, const float** pcm, size_t* floats);
/* Starts a fresh bank at a planning boundary (AudioBank::releaseDecoded). */
int cs_host_release_bank(cs_host* host);

/* PCM16 WAV writer with logical zero padding to `frames` (src/io/audio.cpp:264-285),
 * published atomically through a temporary file in the destination directory. */
int cs_write_wave(const char* path, const int16_t* pcm, int data_frames, int frames, int rate, int channels);
/* True when `path` is a complete PCM16 WAV of this rate and channel count
 * (AudioBank::completeOutput for WAV, src/io/audio.cpp:156-166). */
int cs_wave_complete(const char* path, int rate, int channels);

const char* cs_host_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
