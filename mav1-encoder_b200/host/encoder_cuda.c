/* The mav1 encoder API (src/mav1.h of neolite/mav1-encoder, unchanged) on
 * the B200 encode backend: the Linux host driver.
 *
 * Frames go through the device-resident stream of libmav1cu (every backend
 * stage on the GPU, reference slots in HBM, reference-chain and
 * non-reference frames on two concurrent frame engines). Entropy coding and
 * OBU assembly stay on the host CPU, overlapped with the device: each coded
 * frame's writer inputs are exported into a page-locked image, a poller
 * thread watches the exports complete, and a process-wide pool of worker
 * threads runs the reference's unchanged tile writer on them, a task per
 * tile column (writer.c), then the frame OBU. A frame's image is released to
 * its engine's ring once the tiles are coded; temporal units are assembled
 * in coding order.
 *
 * The frame structure is the reference driver's: the ALTREF queue
 * (mav1_send_frame / alt_drain / pyr_code / alt_code, encoder.c:1004-1320)
 * and the low-delay path (mav1_encode, encoder.c:820-875), planned
 * incrementally by mav1cu_plan_frames. Temporal units follow tu_new /
 * tu_close / tu_show_existing (encoder.c:934-984): a temporal delimiter, the
 * sequence header before a key frame, frame OBUs, closed by a shown frame or
 * a show_existing_frame header, which carries the shown frame's
 * reconstruction for mav1_get_recon. The bitstream, the reconstructions and
 * the MAV1_DUMP_DEC records equal the reference CPU path's.
 *
 * There is no CPU backend: cfg.use_metal = 0 (--cpu) is refused, and so is
 * a machine without the CUDA library or device. */
#include <errno.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "mav1.h"
#include "mav1_cuda.h"
#include "mav1cu.h"
#include "mh_writer.h"

#define JOBRING 64      /* frames between submission and their temporal unit */
#define SRCRING 128     /* source frames by display index */
#define MAX_TILE_COLS 64
#define NUM_ENGINES 2

_Static_assert(sizeof(Mav1Config) == sizeof(mav1cu_config), "Mav1Config layout");

static double now_s(void) {
  struct timespec t;
  clock_gettime(CLOCK_MONOTONIC, &t);
  return t.tv_sec + t.tv_nsec * 1e-9;
}

/* A reconstruction shared by the slots and packets that show it. */
typedef struct {
  atomic_int refs;
  uint8_t data[];
} Recon;

static Recon *recon_ref(Recon *r) {
  if (r) atomic_fetch_add(&r->refs, 1);
  return r;
}
static void recon_unref(Recon *r) {
  if (r && atomic_fetch_sub(&r->refs, 1) == 1) free(r);
}

/* An export image with its writer context: one in-flight frame. */
typedef struct Img {
  uint8_t *image;
  mh_writer *w;
  int engine;
  struct Img *next;
} Img;

typedef struct Job {
  struct Mav1Encoder *enc;
  mav1cu_frame_job job;
  mav1cu_frame_params fp;
  long idx;                 /* coding-order index */
  int engine;
  mav1cu_session *sess;
  int64_t seq;              /* export sequence number on sess */
  Img *img;
  uint8_t *src;             /* page-locked source (back to the pool once the export is complete) */
  int last_hint, arf_hint, ref_hint[7];
  /* entropy coding */
  int ntiles;
  atomic_int tiles_left;
  uint8_t *tile[MAX_TILE_COLS];
  size_t tile_size[MAX_TILE_COLS];
  uint8_t *obu;             /* [sequence header] frame OBU */
  size_t obu_size, tile_bytes;
  uint8_t *dump;
  size_t dump_size;
  Recon *recon;
  Mav1FrameStats st;
  double t0;
  int failed;
  int xstatus;              /* the export header's status when it reported the failure (1 over capacity, 2 invalid blocks) */
  atomic_int state;         /* 0 free, 1 submitted, 2 coded */
} Job;

typedef struct {
  uint8_t *data;
  size_t size;
  Recon *recon;
  Mav1FrameStats st;
} Packet;

/* ---- process-wide entropy pool -------------------------------------------- */

typedef struct Task {
  Job *job;
  int tile;                 /* -1: the frame's set-up */
} Task;

typedef struct Pending {
  Job *job;
  struct Pending *next;
} Pending;

static struct {
  pthread_mutex_t mu;
  pthread_cond_t cv;        /* tasks available / stop */
  pthread_cond_t pcv;       /* pending exports available / stop */
  int users, nthreads, stop;
  pthread_t *th, poller;
  Task *q;                  /* deque of tasks */
  int qcap, qhead, qn;
  Pending *pend_head, *pend_tail, *pend_free;
} pool = {PTHREAD_MUTEX_INITIALIZER, PTHREAD_COND_INITIALIZER, PTHREAD_COND_INITIALIZER};

static void run_task(Task t);

static void q_grow(void) {
  int nc = pool.qcap ? 2 * pool.qcap : 256;
  Task *n = malloc(sizeof(Task) * nc);
  for (int i = 0; i < pool.qn; i++) n[i] = pool.q[(pool.qhead + i) % pool.qcap];
  free(pool.q);
  pool.q = n;
  pool.qcap = nc;
  pool.qhead = 0;
}

/* Tile tasks go to the front (they finish frames already started), frame
 * set-ups to the back. Called with pool.mu held. */
static void q_push(Task t, int front) {
  if (pool.qn == pool.qcap) q_grow();
  if (front) {
    pool.qhead = (pool.qhead + pool.qcap - 1) % pool.qcap;
    pool.q[pool.qhead] = t;
  } else {
    pool.q[(pool.qhead + pool.qn) % pool.qcap] = t;
  }
  pool.qn++;
}

static void *worker(void *arg) {
  (void)arg;
  pthread_mutex_lock(&pool.mu);
  for (;;) {
    while (!pool.stop && pool.qn == 0) pthread_cond_wait(&pool.cv, &pool.mu);
    if (pool.qn == 0 && pool.stop) break;
    Task t = pool.q[pool.qhead];
    pool.qhead = (pool.qhead + 1) % pool.qcap;
    pool.qn--;
    pthread_mutex_unlock(&pool.mu);
    run_task(t);
    pthread_mutex_lock(&pool.mu);
  }
  pthread_mutex_unlock(&pool.mu);
  return NULL;
}

/* Watches the submitted exports and queues a frame's set-up once its image
 * is complete. Exports complete about in submission order; the poller scans
 * the pending list in that order and sleeps briefly when none is ready. */
static void *poller(void *arg) {
  (void)arg;
  pthread_mutex_lock(&pool.mu);
  for (;;) {
    while (!pool.stop && !pool.pend_head) pthread_cond_wait(&pool.pcv, &pool.mu);
    if (pool.stop && !pool.pend_head) break;
    int progressed = 0;
    Pending **pp = &pool.pend_head, *prev = NULL;
    while (*pp) {
      Pending *p = *pp;
      pthread_mutex_unlock(&pool.mu);
      int rc = mav1cu_export_query(p->job->sess, p->job->seq);
      pthread_mutex_lock(&pool.mu);
      if (rc == 0) {
        prev = p;
        pp = &p->next;
        continue;
      }
      if (rc < 0) p->job->failed = rc;
      *pp = p->next;
      if (pool.pend_tail == p) pool.pend_tail = prev;
      p->next = pool.pend_free;
      pool.pend_free = p;
      q_push((Task){p->job, -1}, 0);
      pthread_cond_signal(&pool.cv);
      progressed = 1;
    }
    if (!progressed) {
      pthread_mutex_unlock(&pool.mu);
      struct timespec ts = {0, 20000};
      nanosleep(&ts, NULL);
      pthread_mutex_lock(&pool.mu);
    }
  }
  pthread_mutex_unlock(&pool.mu);
  return NULL;
}

static int pool_threads(void) {
  const char *v = getenv("MAV1_CUDA_THREADS");
  int n = v ? atoi(v) : (int)sysconf(_SC_NPROCESSORS_ONLN);
  return n < 1 ? 1 : n > 256 ? 256 : n;
}

static int pool_acquire(void) {
  pthread_mutex_lock(&pool.mu);
  if (pool.users++ == 0) {
    pool.stop = 0;
    pool.nthreads = pool_threads();
    pool.th = calloc((size_t)pool.nthreads, sizeof(pthread_t));
    for (int i = 0; i < pool.nthreads; i++) pthread_create(&pool.th[i], NULL, worker, NULL);
    pthread_create(&pool.poller, NULL, poller, NULL);
  }
  pthread_mutex_unlock(&pool.mu);
  return 0;
}

static void pool_release(void) {
  pthread_mutex_lock(&pool.mu);
  if (--pool.users > 0) {
    pthread_mutex_unlock(&pool.mu);
    return;
  }
  pool.stop = 1;
  pthread_cond_broadcast(&pool.cv);
  pthread_cond_broadcast(&pool.pcv);
  pthread_mutex_unlock(&pool.mu);
  for (int i = 0; i < pool.nthreads; i++) pthread_join(pool.th[i], NULL);
  pthread_join(pool.poller, NULL);
  free(pool.th);
  pool.th = NULL;
  free(pool.q);
  pool.q = NULL;
  pool.qcap = pool.qn = pool.qhead = 0;
  while (pool.pend_free) {
    Pending *p = pool.pend_free;
    pool.pend_free = p->next;
    free(p);
  }
}

static void pool_pending(Job *j) {
  pthread_mutex_lock(&pool.mu);
  Pending *p = pool.pend_free;
  if (p) pool.pend_free = p->next;
  else p = malloc(sizeof *p);
  p->job = j;
  p->next = NULL;
  if (pool.pend_tail) pool.pend_tail->next = p;
  else pool.pend_head = p;
  pool.pend_tail = p;
  pthread_cond_signal(&pool.pcv);
  pthread_mutex_unlock(&pool.mu);
}

/* ---- the encoder ------------------------------------------------------------ */

struct Mav1Encoder {
  Mav1Config cfg;           /* as given */
  mav1cu_config ccfg;       /* the same bytes, for the C ABI */
  mav1cu_layout L;
  mav1cu_planner pl;
  mav1cu_stream *st;
  int low_delay;
  size_t i420, cap;
  const char *dump_path;
  mh_writer *hw;            /* writer view for mav1_sequence_header */

  pthread_mutex_t mu;
  pthread_cond_t cv;        /* images released, frames written, packets queued */
  Img *free_img[NUM_ENGINES];
  Img *imgs;
  int nimg;
  uint8_t *srcs[SRCRING];   /* by display index */
  uint8_t **src_pool;       /* free page-locked sources */
  int src_pool_n, src_pool_cap, src_count;
  Job jobs[JOBRING];
  long submitted, written;
  int slot_hint[8];
  /* temporal unit being assembled (coding order) */
  uint8_t *tu;
  size_t tu_pos, tu_cap;
  int tu_open;
  Mav1FrameStats tu_st;
  Recon *slot_recon[8];
  Packet *outq;
  int out_n, out_pos, out_cap;
  Recon *shown_recon;
  Mav1FrameStats last;
  int flushing;
  int err;
  char msg[256];
  FILE *dump;
  mav1_cuda_counters counters;  /* under mu */
};

static int fail(struct Mav1Encoder *e, const char *what) {
  if (!e->err) {
    e->err = -1;
    mav1cu_session *s = mav1cu_stream_session(e->st);
    snprintf(e->msg, sizeof e->msg, "%s: %s", what, s ? mav1cu_error_string(s) : "");
    fprintf(stderr, "mav1 (cuda): %s\n", e->msg);
  }
  return -1;
}

void mav1_default_config(Mav1Config *cfg, int width, int height) {
  /* mav1_default_config, encoder.c:51-66 */
  memset(cfg, 0, sizeof(*cfg));
  cfg->width = width;
  cfg->height = height;
  cfg->qindex = 100;
  cfg->use_metal = 1;
  cfg->tx_search = 1;
  cfg->tx_depth = 1;
  cfg->restoration = 1;
  cfg->switchable_interp = 1;
  cfg->intra_edge_filter = 1;
  cfg->loop_filter = 1;
  cfg->cdef = 1;
  cfg->me_range = 32;
}

const char *const mav1_tool_names[16] = {"intra", "inter", "cfl", "angle_delta", "tx_non_dct", "skip",
                                          "rect_part", "compound", "obmc", "lr_wiener_units", "lr_sgr_units",
                                          "golden", "altref", "", "", ""};

static int images_per_engine(void) {
  const char *v = getenv("MAV1_CUDA_IMAGES");
  int n = v ? atoi(v) : 8;
  return n < 1 ? 1 : n > JOBRING / NUM_ENGINES ? JOBRING / NUM_ENGINES : n;
}

Mav1Encoder *mav1_create(const Mav1Config *cfg, char *err, size_t errlen) {
  if (cfg->width < 16 || cfg->height < 16 || cfg->width > 65536 || cfg->height > 65536) {
    snprintf(err, errlen, "unsupported frame size %dx%d", cfg->width, cfg->height);
    return NULL;
  }
  if (!cfg->use_metal) {
    snprintf(err, errlen, "this build encodes on the GPU only (no CPU backend): use_metal must be 1");
    return NULL;
  }
  struct Mav1Encoder *e = calloc(1, sizeof *e);
  e->cfg = *cfg;
  memcpy(&e->ccfg, cfg, sizeof e->ccfg);
  mav1cu_layout_of(&e->ccfg, &e->L);
  e->low_delay = e->L.cfg.altref == 0;
  e->i420 = (size_t)cfg->width * cfg->height + 2 * (size_t)((cfg->width + 1) >> 1) * ((cfg->height + 1) >> 1);
  e->dump_path = getenv("MAV1_DUMP_DEC");
  pthread_mutex_init(&e->mu, NULL);
  pthread_cond_init(&e->cv, NULL);
  if (mav1cu_stream_create(&e->ccfg, &e->st, err, errlen)) {
    free(e);
    return NULL;
  }
  e->cap = mav1cu_export_capacity(mav1cu_stream_engine(e->st, 0));
  e->hw = mh_writer_new(&e->L);
  int per = images_per_engine();
  e->imgs = calloc((size_t)per * NUM_ENGINES, sizeof(Img));
  int ok = e->hw && e->imgs;
  for (int k = 0; ok && k < NUM_ENGINES; k++)
    for (int i = 0; ok && i < per; i++) {
      Img *m = &e->imgs[e->nimg];
      m->engine = k;
      m->image = mav1cu_host_alloc(e->cap);
      m->w = mh_writer_new(&e->L);
      ok = m->image && m->w;
      e->nimg++;
      m->next = e->free_img[k];
      e->free_img[k] = m;
    }
  if (!ok) {
    snprintf(err, errlen, "host allocation of the export images failed (%d of %zu bytes)", per * NUM_ENGINES, e->cap);
    e->err = -1;
    mav1_destroy(e);
    return NULL;
  }
  pool_acquire();
  return e;
}

static uint8_t *src_get(struct Mav1Encoder *e) {
  pthread_mutex_lock(&e->mu);
  uint8_t *p = e->src_pool_n ? e->src_pool[--e->src_pool_n] : NULL;
  pthread_mutex_unlock(&e->mu);
  if (!p) {
    p = mav1cu_host_alloc(e->i420);
    if (p) {
      pthread_mutex_lock(&e->mu);
      e->src_count++;
      pthread_mutex_unlock(&e->mu);
    }
  }
  return p;
}

/* called with e->mu held */
static void src_put(struct Mav1Encoder *e, uint8_t *p) {
  if (!p) return;
  if (e->src_pool_n == e->src_pool_cap) {
    e->src_pool_cap = e->src_pool_cap ? 2 * e->src_pool_cap : 16;
    e->src_pool = realloc(e->src_pool, sizeof(uint8_t *) * e->src_pool_cap);
  }
  e->src_pool[e->src_pool_n++] = p;
}

/* ---- temporal units (coding order, under e->mu) ---------------------------- */

static void tu_reserve(struct Mav1Encoder *e, size_t n) {
  if (e->tu_pos + n > e->tu_cap) {
    e->tu_cap = (e->tu_pos + n) * 2;
    e->tu = realloc(e->tu, e->tu_cap);
  }
}

static void tu_open(struct Mav1Encoder *e, int frameType) {
  e->tu = NULL;
  e->tu_pos = e->tu_cap = 0;
  tu_reserve(e, 1024);
  e->tu_pos = mh_temporal_delimiter(e->tu);
  memset(&e->tu_st, 0, sizeof e->tu_st);
  e->tu_st.frame_type = frameType;
  e->tu_open = 1;
}

static void tu_close(struct Mav1Encoder *e, Recon *r) {
  if (e->out_n == e->out_cap) {
    e->out_cap = e->out_cap ? 2 * e->out_cap : 16;
    e->outq = realloc(e->outq, sizeof(Packet) * e->out_cap);
  }
  Packet *p = &e->outq[e->out_n++];
  p->data = e->tu;
  p->size = e->tu_pos;
  p->recon = recon_ref(r);
  p->st = e->tu_st;
  p->st.bytes = e->tu_pos;
  e->tu = NULL;
  e->tu_pos = e->tu_cap = 0;
  e->tu_open = 0;
}

static void stats_add(Mav1FrameStats *a, const Mav1FrameStats *b) {
  a->num_blocks += b->num_blocks;
  a->num_inter_blocks += b->num_inter_blocks;
  for (int k = 0; k < 16; k++) a->tool_use[k] += b->tool_use[k];
  a->t_analysis += b->t_analysis;
  a->t_recon += b->t_recon;
  a->t_filter += b->t_filter;
  a->t_entropy += b->t_entropy;
}

/* Appends the coded frames that are next in coding order to the temporal
 * units (alt_code's writer-queue step, encoder.c:1194-1224). */
static void write_ready(struct Mav1Encoder *e) {
  for (;;) {
    Job *j = &e->jobs[e->written % JOBRING];
    if (e->written == e->submitted || atomic_load(&j->state) != 2) break;
    if (j->failed && !e->err) {
      e->err = j->failed;
      /* what failed: the export's own checks, or a kernel's status word (the
       * session's synchronize turns that into its message) */
      const char *why = "";
      if (j->xstatus == 1) why = "the export image's capacity was exceeded";
      else if (j->xstatus == 2) why = "the export found blocks out of range";
      else if (j->failed == MAV1CU_ERR_DEVICE && mav1cu_synchronize(j->sess) != MAV1CU_OK)
        why = mav1cu_error_string(j->sess);
      snprintf(e->msg, sizeof e->msg, "frame %d: device error %d%s%s", j->job.disp, j->failed, *why ? ": " : "", why);
      fprintf(stderr, "mav1 (cuda): %s\n", e->msg);
    }
    if (!e->tu_open) tu_open(e, j->job.is_key ? 0 : 1);
    tu_reserve(e, j->obu_size);
    if (j->obu_size) memcpy(e->tu + e->tu_pos, j->obu, j->obu_size);
    e->tu_pos += j->obu_size;
    stats_add(&e->tu_st, &j->st);
    if (j->dump && e->dump_path) {
      if (!e->dump) e->dump = fopen(e->dump_path, "wb");
      if (e->dump) {
        fwrite(j->dump, 1, j->dump_size, e->dump);
        fflush(e->dump);
      }
    }
    int rf = j->job.refresh;
    for (int k = 0; k < 8; k++)
      if ((rf >> k) & 1) {
        recon_unref(e->slot_recon[k]);
        e->slot_recon[k] = recon_ref(j->recon);
      }
    if (e->low_delay || !j->job.hidden) tu_close(e, j->recon);
    if (!e->low_delay && j->job.show_existing >= 0) {
      if (!e->tu_open) tu_open(e, 1);
      tu_reserve(e, 64);
      e->tu_pos += mh_show_existing(j->job.show_existing, e->tu + e->tu_pos);
      tu_close(e, e->slot_recon[j->job.show_existing]);
    }
    free(j->obu);
    free(j->dump);
    recon_unref(j->recon);
    j->obu = j->dump = NULL;
    j->recon = NULL;
    atomic_store(&j->state, 0);
    e->written++;
  }
  pthread_cond_broadcast(&e->cv);
}

/* ---- entropy tasks ------------------------------------------------------------ */

static void release_and_write(Job *j) {
  struct Mav1Encoder *e = j->enc;
  pthread_mutex_lock(&e->mu);
  Img *m = j->img;
  m->next = e->free_img[m->engine];
  e->free_img[m->engine] = m;
  j->img = NULL;
  atomic_store(&j->state, 2);
  write_ready(e);
  pthread_mutex_unlock(&e->mu);
}

/* A frame whose export failed: nothing is coded; the encoder reports the
 * error when the frame's turn comes. */
static void frame_failed(Job *j) {
  j->obu = NULL;
  j->obu_size = 0;
  j->recon = calloc(1, sizeof(Recon) + j->enc->i420);
  if (j->recon) atomic_init(&j->recon->refs, 1);
  release_and_write(j);
}

static void frame_done(Job *j) {
  struct Mav1Encoder *e = j->enc;
  mh_writer *w = j->img->w;
  size_t total = 0;
  for (int i = 0; i < j->ntiles; i++) total += j->tile_size[i] + (i < j->ntiles - 1 ? 4 : 0);
  /* tile data: every tile but the last preceded by tile_size_minus_1 as
   * le(4) (tile_writer.c:611-623) */
  uint8_t *tile = malloc(total ? total : 1), *q = tile;
  for (int i = 0; i < j->ntiles; i++) {
    if (i < j->ntiles - 1) {
      uint32_t m1 = (uint32_t)j->tile_size[i] - 1;
      for (int b = 0; b < 4; b++) *q++ = (uint8_t)(m1 >> (8 * b));
    }
    memcpy(q, j->tile[i], j->tile_size[i]);
    q += j->tile_size[i];
    free(j->tile[i]);
    j->tile[i] = NULL;
  }
  j->tile_bytes = total;
  j->obu = malloc(total + 2048);
  size_t pos = 0;
  if (j->job.is_key) pos += mh_writer_sequence_header(w, j->obu);
  pos += mh_writer_frame_obu(w, tile, total, j->obu + pos);
  j->obu_size = pos;
  free(tile);
  if (e->dump_path) j->dump = mh_writer_dump_record(w, total, &j->dump_size);
  mh_writer_stats(w, &j->st.num_blocks, &j->st.num_inter_blocks, j->st.tool_use);
  {
    /* the LR search's unit counts (lr_select, lr_search.c:350-351) */
    const mav1cu_export_header *hx = (const mav1cu_export_header *)j->img->image;
    const mav1cu_lr_unit *lu = (const mav1cu_lr_unit *)(j->img->image + hx->lr_off);
    for (int k = 0; k < hx->lr_units; k++) {
      j->st.tool_use[9] += lu[k].type == 1;  /* RESTORE_WIENER */
      j->st.tool_use[10] += lu[k].type == 2; /* RESTORE_SGRPROJ */
    }
  }
  /* the reconstruction section holds the picture as mav1_get_recon returns it */
  const mav1cu_export_header *h = (const mav1cu_export_header *)j->img->image;
  j->recon = malloc(sizeof(Recon) + e->i420);
  atomic_init(&j->recon->refs, 1);
  if (h->rec_bytes == (int64_t)e->i420) memcpy(j->recon->data, j->img->image + h->rec_off, e->i420);
  else memset(j->recon->data, 0, e->i420);
  j->st.frame_type = j->job.is_key ? 0 : 1;
  j->st.t_entropy = now_s() - j->t0;
  pthread_mutex_lock(&e->mu);
  e->counters.frames++;
  e->counters.d2h_bytes += h->bytes;
  e->counters.entropy_s += j->st.t_entropy;
  pthread_mutex_unlock(&e->mu);
  release_and_write(j);
}

static void run_task(Task t) {
  Job *j = t.job;
  struct Mav1Encoder *e = j->enc;
  if (t.tile < 0) {
    /* the export is complete: its upload is too, so the source is free */
    j->t0 = now_s();
    pthread_mutex_lock(&e->mu);
    src_put(e, j->src);
    j->src = NULL;
    pthread_mutex_unlock(&e->mu);
    const mav1cu_export_header *h = (const mav1cu_export_header *)j->img->image;
    if (j->failed || h->status != 0 || h->seq != (int32_t)j->seq) {
      if (!j->failed) {
        j->failed = h->status ? MAV1CU_ERR_DEVICE : MAV1CU_ERR_ARG;
        j->xstatus = h->status;
      }
      frame_failed(j);
      return;
    }
    const uint8_t *img = j->img->image;
    /* the frame's parameters as the device used them: lr_type is the loop-
     * restoration search's */
    memcpy(&j->fp, img + h->params_off, sizeof j->fp);
    mh_frame f = {&j->job, &j->fp, e->low_delay, j->last_hint, j->arf_hint, {0},
                  (const mav1cu_sb_info *)(img + h->sbs_off), (const mav1cu_block_info *)(img + h->blocks_off),
                  (const int32_t *)(img + h->coefs_off), (const int8_t *)(img + h->cdef_off),
                  h->lr_units > 0 ? (const mav1cu_lr_unit *)(img + h->lr_off) : NULL};
    memcpy(f.ref_hint, j->ref_hint, sizeof f.ref_hint);
    mh_writer_frame(j->img->w, &f);
    mh_writer_begin(j->img->w);
    j->ntiles = mh_writer_tile_cols(j->img->w);
    atomic_store(&j->tiles_left, j->ntiles);
    if (j->ntiles > 1) {
      pthread_mutex_lock(&pool.mu);
      for (int tc = j->ntiles - 1; tc >= 1; tc--) q_push((Task){j, tc}, 1);
      pthread_cond_broadcast(&pool.cv);
      pthread_mutex_unlock(&pool.mu);
    }
    t.tile = 0;
  }
  j->tile_size[t.tile] = mh_writer_tile(j->img->w, t.tile, &j->tile[t.tile]);
  if (atomic_fetch_sub(&j->tiles_left, 1) == 1) frame_done(j);
}

/* ---- submission ------------------------------------------------------------ */

static int submit(struct Mav1Encoder *e, const mav1cu_frame_job *job) {
  int rf = job->is_key ? 0xFF : job->refresh;
  int ei = rf ? 0 : 1;  /* the stream's engine split */
  pthread_mutex_lock(&e->mu);
  while (!e->free_img[ei] || e->submitted - e->written >= JOBRING) pthread_cond_wait(&e->cv, &e->mu);
  Img *m = e->free_img[ei];
  e->free_img[ei] = m->next;
  Job *j = &e->jobs[e->submitted % JOBRING];
  pthread_mutex_unlock(&e->mu);
  memset(j, 0, sizeof *j);
  j->enc = e;
  j->job = *job;
  j->idx = e->submitted;
  j->engine = ei;
  j->img = m;
  j->src = e->srcs[job->disp % SRCRING];
  e->srcs[job->disp % SRCRING] = NULL;
  int presets = 0;
  mav1cu_frame_params_for(&e->ccfg, job, &j->fp, &presets);
  if (e->low_delay) {
    /* MAV1_DUMP_DEC hints of mav1_encode (encoder.c:837-838) */
    j->last_hint = job->is_key ? -1 : job->order_hint - 1 - (e->L.cfg.nonref_odd && (job->order_hint & 1) == 0 ? 1 : 0);
    j->arf_hint = -1;
  } else {
    j->last_hint = job->is_key ? -1 : e->slot_hint[job->last_slot];
    j->arf_hint = !job->is_key && job->arf_slot >= 0 ? e->slot_hint[job->arf_slot] : -1;
    for (int i = 0; i < 7; i++) {
      int slot = i == 6 && job->arf_slot >= 0 ? job->arf_slot : job->last_slot;
      j->ref_hint[i] = job->is_key ? 0 : e->slot_hint[slot];
    }
    for (int k = 0; k < 8; k++)
      if ((rf >> k) & 1) e->slot_hint[k] = job->order_hint;
  }
  if (!j->src) return fail(e, "source frame missing");
  if (mav1cu_stream_encode(e->st, job, j->src, 0)) return fail(e, "stream encode");
  j->sess = mav1cu_stream_engine(e->st, ei);
  if (mav1cu_export(j->sess, m->image, e->cap, MAV1CU_EXPORT_REC | (e->L.cfg.restoration ? MAV1CU_EXPORT_LR : 0)))
    return fail(e, "export");
  j->seq = mav1cu_export_seq(j->sess);
  atomic_store(&j->state, 1);
  pthread_mutex_lock(&e->mu);
  e->counters.h2d_bytes += (int64_t)e->i420;
  e->submitted++;
  pthread_mutex_unlock(&e->mu);
  pool_pending(j);
  return 0;
}

static int plan_and_submit(struct Mav1Encoder *e, int newFrames, int flush) {
  mav1cu_frame_job jobs[64];
  int n = mav1cu_plan_frames(&e->ccfg, &e->pl, newFrames, flush, jobs, 64);
  if (n < 0) return fail(e, "planning");
  for (int i = 0; i < n; i++)
    if (submit(e, &jobs[i])) return -1;
  return 0;
}

int mav1_send_frame(Mav1Encoder *e, const uint8_t *const planes[3], const int strides[3]) {
  if (e->err) return e->err;
  if (!planes) {
    if (e->flushing) return 0;
    e->flushing = 1;
    return plan_and_submit(e, 0, 1);
  }
  /* packs the input (mav1_send_frame, encoder.c:1302-1311) into page-locked
   * memory for the asynchronous upload */
  uint8_t *f = src_get(e);
  if (!f) return fail(e, "source allocation");
  int w = e->cfg.width, h = e->cfg.height, cw = (w + 1) >> 1, ch = (h + 1) >> 1;
  for (int p = 0; p < 3; p++) {
    int pw = p ? cw : w, ph = p ? ch : h;
    uint8_t *d = f + (p ? (size_t)w * h + (p - 1) * (size_t)cw * ch : 0);
    for (int y = 0; y < ph; y++) memcpy(d + (size_t)y * pw, planes[p] + (size_t)y * strides[p], pw);
  }
  int disp = e->pl.in_disp;
  if (e->srcs[disp % SRCRING]) return fail(e, "too many queued source frames");
  e->srcs[disp % SRCRING] = f;
  if (plan_and_submit(e, 1, 0)) return -1;
  if (e->low_delay) {
    /* mav1_encode is synchronous: its packet is ready when send returns */
    pthread_mutex_lock(&e->mu);
    while (e->written < e->submitted && !e->err) pthread_cond_wait(&e->cv, &e->mu);
    pthread_mutex_unlock(&e->mu);
  }
  return e->err;
}

int mav1_encode(Mav1Encoder *e, const uint8_t *const planes[3], const int strides[3], uint8_t **out,
                size_t *outSize) {
  if (!e->low_delay) {
    snprintf(e->msg, sizeof e->msg, "mav1_encode needs a configuration without ALTREF (use the queue API)");
    return -1;
  }
  if (mav1_send_frame(e, planes, strides)) return -1;
  return mav1_receive_packet(e, out, outSize) ? -1 : 0;
}

/* called with e->mu held */
static int pop_packet(struct Mav1Encoder *e, uint8_t **out, size_t *outSize) {
  if (e->out_pos == e->out_n) {
    e->out_pos = e->out_n = 0;
    return 1;
  }
  Packet p = e->outq[e->out_pos++];
  *out = p.data;
  *outSize = p.size;
  recon_unref(e->shown_recon);
  e->shown_recon = p.recon;
  e->last = p.st;
  return 0;
}

int mav1_receive_packet(Mav1Encoder *e, uint8_t **out, size_t *outSize) {
  pthread_mutex_lock(&e->mu);
  /* when flushing, every queued frame is waited for */
  if (e->flushing)
    while (e->written < e->submitted) pthread_cond_wait(&e->cv, &e->mu);
  int rc = pop_packet(e, out, outSize);
  pthread_mutex_unlock(&e->mu);
  return rc;
}

int mav1_busy(Mav1Encoder *e) {
  pthread_mutex_lock(&e->mu);
  int b = e->pl.inq_n > 0 || e->written < e->submitted;
  pthread_mutex_unlock(&e->mu);
  return b;
}

int mav1_pending_packets(Mav1Encoder *e) {
  pthread_mutex_lock(&e->mu);
  int n = e->out_n - e->out_pos;
  pthread_mutex_unlock(&e->mu);
  return n;
}

int mav1_receive_packet_wait(Mav1Encoder *e, uint8_t **out, size_t *outSize, int timeout_ms) {
  /* encoder.c:1362-1396: while flushing, work in flight may outlast the
   * timeout; the timeout bounds polls of a live stream only */
  struct timespec ts;
  clock_gettime(CLOCK_REALTIME, &ts);
  ts.tv_nsec += (long)timeout_ms * 1000000;
  ts.tv_sec += ts.tv_nsec / 1000000000;
  ts.tv_nsec %= 1000000000;
  pthread_mutex_lock(&e->mu);
  for (;;) {
    if (e->out_pos != e->out_n) break;
    if (e->written == e->submitted && (e->flushing || e->err)) break;
    if (pthread_cond_timedwait(&e->cv, &e->mu, &ts) == ETIMEDOUT) {
      if (!e->flushing || e->written == e->submitted) break;
      clock_gettime(CLOCK_REALTIME, &ts);
      ts.tv_nsec += (long)timeout_ms * 1000000;
      ts.tv_sec += ts.tv_nsec / 1000000000;
      ts.tv_nsec %= 1000000000;
    }
  }
  int rc = pop_packet(e, out, outSize);
  pthread_mutex_unlock(&e->mu);
  return rc;
}

size_t mav1_sequence_header(const Mav1Encoder *e, uint8_t *out) { return mh_writer_sequence_header(e->hw, out); }

void mav1_get_recon(const Mav1Encoder *e, uint8_t *const planes[3], const int strides[3]) {
  const Recon *r = e->shown_recon;
  if (!r) return;
  int w = e->cfg.width, h = e->cfg.height, cw = (w + 1) >> 1, ch = (h + 1) >> 1;
  const uint8_t *src[3] = {r->data, r->data + (size_t)w * h, r->data + (size_t)w * h + (size_t)cw * ch};
  for (int p = 0; p < 3; p++) {
    int pw = p ? cw : w, ph = p ? ch : h;
    for (int y = 0; y < ph; y++) memcpy(planes[p] + (size_t)y * strides[p], src[p] + (size_t)y * pw, pw);
  }
}

const Mav1FrameStats *mav1_last_stats(const Mav1Encoder *e) { return &e->last; }

int64_t mav1_cuda_device_bytes(const Mav1Encoder *e) { return mav1cu_stream_device_bytes(e->st); }

int mav1_cuda_restart(Mav1Encoder *e, const Mav1Config *cfg) {
  if (cfg->width != e->cfg.width || cfg->height != e->cfg.height || !cfg->use_metal) return -1;
  pthread_mutex_lock(&e->mu);
  while (e->written < e->submitted) pthread_cond_wait(&e->cv, &e->mu);
  pthread_mutex_unlock(&e->mu);
  mav1cu_config c;
  memcpy(&c, cfg, sizeof c);
  if (mav1cu_stream_reconfigure(e->st, &c)) return fail(e, "restart");
  e->cfg = *cfg;
  e->ccfg = c;
  mav1cu_layout_of(&e->ccfg, &e->L);
  e->low_delay = e->L.cfg.altref == 0;
  mh_writer_config(e->hw, &e->L);
  for (int i = 0; i < e->nimg; i++) mh_writer_config(e->imgs[i].w, &e->L);
  memset(&e->pl, 0, sizeof e->pl);
  pthread_mutex_lock(&e->mu);
  for (int i = 0; i < SRCRING; i++)
    if (e->srcs[i]) {
      src_put(e, e->srcs[i]);
      e->srcs[i] = NULL;
    }
  pthread_mutex_unlock(&e->mu);
  for (int i = e->out_pos; i < e->out_n; i++) {
    free(e->outq[i].data);
    recon_unref(e->outq[i].recon);
  }
  e->out_pos = e->out_n = 0;
  free(e->tu);
  e->tu = NULL;
  e->tu_pos = e->tu_cap = 0;
  e->tu_open = 0;
  for (int k = 0; k < 8; k++) {
    recon_unref(e->slot_recon[k]);
    e->slot_recon[k] = NULL;
  }
  memset(e->slot_hint, 0, sizeof e->slot_hint);
  recon_unref(e->shown_recon);
  e->shown_recon = NULL;
  memset(&e->last, 0, sizeof e->last);
  e->flushing = 0;
  return 0;
}

int64_t mav1_cuda_device_bytes_for(const Mav1Config *cfg) {
  mav1cu_config c;
  memcpy(&c, cfg, sizeof c);
  return mav1cu_stream_bytes_for(&c);
}

void mav1_cuda_get_counters(const Mav1Encoder *e, mav1_cuda_counters *out) {
  pthread_mutex_lock((pthread_mutex_t *)&e->mu);
  *out = e->counters;
  pthread_mutex_unlock((pthread_mutex_t *)&e->mu);
}
const char *mav1_backend_name(const Mav1Encoder *e) {
  (void)e;
  return "cuda-sm_100a";
}

void mav1_destroy(Mav1Encoder *e) {
  if (!e) return;
  if (e->st) {
    /* frames in flight finish their entropy coding first */
    pthread_mutex_lock(&e->mu);
    while (e->written < e->submitted) pthread_cond_wait(&e->cv, &e->mu);
    pthread_mutex_unlock(&e->mu);
    mav1cu_stream_synchronize(e->st);
    pool_release();
    mav1cu_stream_destroy(e->st);
  }
  for (int i = 0; i < e->nimg; i++) {
    mav1cu_host_free(e->imgs[i].image);
    mh_writer_free(e->imgs[i].w);
  }
  free(e->imgs);
  mh_writer_free(e->hw);
  for (int i = 0; i < SRCRING; i++) mav1cu_host_free(e->srcs[i]);
  for (int i = 0; i < e->src_pool_n; i++) mav1cu_host_free(e->src_pool[i]);
  free(e->src_pool);
  for (int i = e->out_pos; i < e->out_n; i++) {
    free(e->outq[i].data);
    recon_unref(e->outq[i].recon);
  }
  free(e->outq);
  free(e->tu);
  for (int k = 0; k < 8; k++) recon_unref(e->slot_recon[k]);
  recon_unref(e->shown_recon);
  if (e->dump) fclose(e->dump);
  pthread_mutex_destroy(&e->mu);
  pthread_cond_destroy(&e->cv);
  free(e);
}
