/*
 * n3: B200-native (sm_100a) engine for the no-three-in-line population search.
 *
 * Flat C ABI of libn3.so.  Every entry point takes device pointers (caller
 * owned), plain sizes and a CUDA stream (cudaStream_t passed as void*; NULL is
 * the legacy default stream), enqueues its work on that stream and returns an
 * int status: N3_OK (0) or one of the N3_ERR_* codes below.  The message of
 * the last failure on the calling host thread is returned by n3_last_error().
 * Calls that report device-side findings (mismatch counts, error words) write
 * them to device memory; read them after synchronising the stream.
 *
 * State layout: the reference's interleaved slot layout
 * (src/no_three_75/accelerated.py:18-24, src/no_three_75/tempering.py:38).
 * A state of an n x n grid has m = 2n slots; slot s = 2*row + layer lies in row
 * s >> 1 and its column is cols[s].  P/Q arrays ([B][n] int32, the layout of
 * src/no_three_75/gpu.py:69-77) are accepted where the reference used them.
 * Columns must lie in [0, n); 2 <= n <= N3_MAX_N.
 *
 * Energies are exact integers everywhere: E = number of collinear triples.
 */
#ifndef N3_H_
#define N3_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define N3_MAX_N 75
#define N3_SENTINEL (1 << 30) /* illegal move marker, src/no_three_75/gpu_delta.py:35 */

enum {
  N3_OK = 0,
  N3_ERR_ARG = 1,      /* null pointer, bad size or shape (reference: ValueError) */
  N3_ERR_RANGE = 2,    /* n outside [2, N3_MAX_N] or an index out of range */
  N3_ERR_CUDA = 3,     /* CUDA runtime failure or no device (reference: RuntimeError) */
  N3_ERR_MISMATCH = 4, /* incremental / cross-checked count differs (reference: AssertionError) */
  N3_ERR_TIMEOUT = 5,  /* a bounded device wait expired */
  N3_ERR_STATE = 6     /* the state is not a legal two-per-row/column state */
};

/* Library version (major*10000 + minor*100 + patch). */
int n3_version(void);

/* Message of the last failing call on this host thread ("" if none). */
const char* n3_last_error(void);

/* One-time set-up on the current device: builds the device-resident tables
 * and opts the kernels into their shared-memory carve-outs.  Every entry
 * point does what it needs of this lazily; call it once first when the
 * first launches on a device are to be captured into a CUDA graph. */
int n3_init_device(void);

/* ---------------------------------------------------------------------------
 * (a) Population scoring.
 * ------------------------------------------------------------------------- */

/* Exact collinear-triple count of B states given as P/Q, one warp per state,
 * int32 cross-product determinants.  Replaces the reference kernel
 * score_population (src/no_three_75/gpu.py:13-42, launched at gpu.py:76) and,
 * with badness != NULL, score_population_badness
 * (src/no_three_75/gpu_device_search.py:118-161): badness[b][s] is the number
 * of collinear triples containing slot s.
 *   p, q     int32 [B][n]      scores int32 [B]      badness int32 [B][2n] or NULL */
int n3_score_population(const int32_t* p, const int32_t* q, int B, int n, int32_t* scores,
                        int32_t* badness, void* stream);

/* Same count over slot-layout columns (int16 [B][2n]). */
int n3_score_columns(const int16_t* cols, int B, int n, int32_t* scores, int32_t* badness,
                     void* stream);

/* Independent normalised-slope line count: for each anchor the other points
 * are grouped by gcd-reduced undirected direction (src/no_three_75/verifier_b.py:8-19);
 * badness[s] = sum over directions of C(c,2) (src/no_three_75/conflicts.py:376-378)
 * and E = sum(badness)/3 = sum over lines of C(k,3) (conflicts.py:373).
 *   cols int16 [B][2n]     scores int32 [B]     badness int32 [B][2n] or NULL */
int n3_score_slope(const int16_t* cols, int B, int n, int32_t* scores, int32_t* badness,
                   void* stream);

/* Fused, cross-checked scoring: determinant count and slope count per state,
 * plus the column-range / duplicate-point checks.  scores = determinant E,
 * badness = slope badness, or NULL: then the slope side counts E alone, each
 * collinear triple once from its first slot (about 2/3 of the slope side's
 * time).  *mismatch (device int32, accumulated, caller zeroes it) counts
 * states whose two counts differ or whose badness does not sum to 3E;
 * *error_word (device uint32, OR-ed, caller zeroes it, may be NULL) collects
 * the device error bits (1: column range, 2: duplicate point, 4: mismatch).  The reference runs this audit on the host
 * (src/no_three_75/gpu.py:131 exact_match, src/no_three_75/tempering.py:193-204). */
int n3_score_checked(const int16_t* cols, int B, int n, int32_t* scores, int32_t* badness,
                     int32_t* mismatch, uint32_t* error_word, void* stream);

/* ---------------------------------------------------------------------------
 * (b) Exact incremental swap deltas.
 *
 * A move (state, u, v) exchanges the columns of slots u and v (different
 * rows); it is legal iff the columns differ and neither new point duplicates
 * the other point of its row (src/no_three_75/tempering.py:58).  Illegal moves
 * and out-of-range indices give N3_SENTINEL.
 * ------------------------------------------------------------------------- */

/* Exact dE of each move, counted through the moved points only (direction
 * classes around u, v and their new positions); bit-exact against a full
 * recompute.  Replaces the per-proposal delta of the reference walk kernel
 * (src/no_three_75/tempering.py:68-89) for batches of moves.
 *   cols int16 [B][2n]   moves int32 [M][3] (state, u, v)   dE int32 [M]
 *   dbad int32 [M][2n] or NULL: change of every slot's badness (slot u / v
 *   refer to the moved points' new positions). */
int n3_swap_delta(const int16_t* cols, int B, int n, const int32_t* moves, int M, int32_t* dE,
                  int32_t* dbad, void* stream);

/* Same result by the reference's literal formulation (tempering.py:68-89:
 * every pair outside {u,v} tested against u, u', v, v', every k against
 * (u,v) and (u',v')); an independent device cross-check of n3_swap_delta. */
int n3_swap_delta_pairs(const int16_t* cols, int B, int n, const int32_t* moves, int M,
                        int32_t* dE, int32_t* dbad, void* stream);

/* Full score after exchanging anchor slot u with every partner slot v, for A
 * anchors (state, u): out[a][v] = current[state] - (bad[u] + bad[v] - joint)
 * + new_affected, N3_SENTINEL where illegal.  Replaces the reference plugin
 * kernel two_switch_scores (src/no_three_75/gpu_delta.py:19-75, one anchor per
 * launch at gpu_delta.py:103-115) and accelerated.evaluate_two_switches
 * (src/no_three_75/accelerated.py:122-195).
 *   badness int32 [B][2n]   current int32 [B]   anchors int32 [A][2]   out int32 [A][2n] */
int n3_two_switch_scores(const int16_t* cols, const int32_t* badness, const int32_t* current,
                         int B, int n, const int32_t* anchors, int A, int32_t* out, void* stream);

/* Same-layer row transpositions of anchor slot u = 2*row + layer with every
 * partner row: out[a][row'] (int32 [A][n]), N3_SENTINEL where illegal or
 * row' == row.  Replaces accelerated.evaluate_transpositions
 * (src/no_three_75/accelerated.py:40-119). */
int n3_transposition_scores(const int16_t* cols, const int32_t* badness, const int32_t* current,
                            int B, int n, const int32_t* anchors, int A, int32_t* out, void* stream);

/* ---------------------------------------------------------------------------
 * (c) Replica-exchange tempering.
 *
 * Chains are grouped in ladders of L consecutive chains; chain c belongs to
 * ladder c / L.  Every array below is device memory owned by the caller
 * (the Python TemperingChains object); the kernel keeps each chain's state in
 * shared memory for the whole launch and writes it back at the end.
 * Replaces the reference's walk kernel and TemperingChains.advance/exchange
 * (src/no_three_75/tempering.py:29-191), with the exchange on the device.
 * ------------------------------------------------------------------------- */

#define N3_SLOT_STRIDE 150 /* row stride of the per-chain arrays (2 * N3_MAX_N) */

typedef struct n3_chains {
  int n_chains;                 /* C, a positive multiple of ladder_size */
  int ladder_size;              /* L, temperatures per ladder, 2..64 */
  int16_t* cols;                /* [C][150] slot columns (first 2n used) */
  int32_t* badness;             /* [C][150] triples through each slot, kept exact */
  int32_t* energy;              /* [C] current E */
  int32_t* best_energy;         /* [C] lowest E seen */
  int16_t* best_cols;           /* [C][150] state at best_energy */
  int32_t* temp_of;             /* [C] temperature index of chain c (ladder-major) */
  int32_t* chain_at;            /* [C] chain_at[l*L + t]: ladder-local chain at temperature t */
  uint64_t* counter;            /* [C] proposals made (Philox counter) */
  uint32_t* accepted;           /* [C] accepted proposals */
  const int32_t* ladder_n;      /* [C/L] grid size n of each ladder (mixed sizes allowed) */
  uint32_t* ladder_round;       /* [C/L] exchange rounds done (even/odd parity) */
  uint32_t* ladder_exchanges;   /* [C/L] accepted exchanges */
  const uint32_t* acc_thresh;   /* [L][acc_width]: accept dE > 0 iff u32 < acc_thresh[t][dE] */
  int acc_width;                /* dE >= acc_width is rejected */
  const uint32_t* exch_thresh;  /* [L-1][exch_width]: swap (t,t+1) with energy gap -d iff u32 < thr[t][d] */
  int exch_width;
  int32_t* global_best;         /* [1] atomic minimum of best_energy, or NULL */
  int32_t* hit;                 /* [4] first chain with E <= target: chain, counter, globaltimer lo/hi; or NULL */
  int32_t* stop;                /* [1] nonzero: stop at the next exchange boundary; or NULL */
  uint32_t* error_word;         /* [1] device error bits (16: incremental/full mismatch); or NULL */
  /* Umbrella restraint on the distance to a reference state
   * (src/no_three_75/tempering.py:57-63, 91-97).  NULL umbrella: no restraint. */
  const int16_t* reference;     /* [150] slot columns of the reference state (rows as in cols) */
  int32_t* removed;             /* [C] reference points missing from chain c, kept exact; NULL without umbrella */
  const int64_t* umbrella;      /* [C][2] per replica position l*L+t: round(2^24 s), round(2^24 * 2 s center) */
  const uint32_t* acc_frac;     /* [L][768] fraction factors floor(2^32 exp(-k/(2^j T))), j = 8, 16, 24, k < 256 */
} n3_chains;

typedef struct n3_temper_config {
  uint64_t seed;                /* Philox key */
  int chains_per_block;         /* warps (chains) per CTA: divides L (cluster of L/cpb CTAs) or a multiple of L */
  int rounds;                   /* exchange rounds this launch (when ladder_rounds is NULL) */
  const int32_t* ladder_rounds; /* [C/L] per-ladder rounds (device), equal within a CTA or cluster; or NULL */
  int round_sweeps;             /* proposals per round = round_sweeps * 2n (one sweep = 2n proposals) ... */
  int round_proposals;          /* ... unless round_proposals > 0 */
  int exchange;                 /* 1: neighbour exchange after every round */
  int target_energy;            /* >= 0: record the first chain reaching E <= target (and raise *stop) */
  int bad_bias;                 /* percent of proposals whose slot u is drawn by badness (tempering.py:51-55) */
  int threads_per_chain;        /* 32 (or 0), 64, 128 or 256: warps that evaluate one chain's moves together;
                                   chains_per_block x threads_per_chain / 32 <= 16 warps per CTA */
} n3_temper_config;

/* Runs cfg->rounds rounds (proposals, then an exchange) on every ladder in one
 * persistent launch: grid C/cpb CTAs of cpb x threads_per_chain threads,
 * clusters of L/cpb CTAs when a ladder spans several CTAs.  Results do not
 * depend on cpb or threads_per_chain (the same proposals, dE and acceptances).  Capturable in a CUDA graph (fixed
 * arguments; the per-device tables must have been set up by an earlier call).
 *
 * A proposal is the reference walk's (tempering.py:49-58): slot u uniform, or,
 * with probability bad_bias/100 while E > 0, drawn in proportion to badness
 * (the first slot whose running badness sum exceeds a uniform integer below
 * 3E); slot v uniform; legal iff E > 0 and the swap duplicates no point.
 * With chains->umbrella set, the acceptance energy adds the reference's
 * restraint s ((removed - center + dd)^2 - (removed - center)^2) in units of
 * 2^-24 (tempering.py:93-94), and an accepted move updates removed by dd.
 * The reference disables exchanges under an umbrella (tempering.py:173-174):
 * so does n3_temper_run (N3_ERR_ARG when exchange is requested). */
int n3_temper_run(const n3_chains* chains, const n3_temper_config* config, void* stream);

/* Recomputes every chain's E (determinant count) and badness (slope count)
 * and adds the number of chains that differ from the maintained values to
 * *mismatch (device int32).  The reference's TemperingChains.validate
 * (src/no_three_75/tempering.py:193-204), on the device. */
int n3_temper_audit(const n3_chains* chains, int32_t* mismatch, void* stream);

/* ---------------------------------------------------------------------------
 * (d) Learned move proposal (no reference counterpart: the reference's walk
 * proposes uniformly, src/no_three_75/tempering.py:50-56).
 *
 * A 192 -> 256 -> 256 -> 1 MLP (ReLU) with bf16 tensor-core weights and fp32
 * accumulation ranks 128 candidate swaps per chain per step by predicted dE;
 * one candidate is drawn from softmax(-pred / T) and accepted with the exact
 * integer delta and the chain's Metropolis thresholds.  Every step pushes the
 * chosen candidate's (features, exact dE) to a ring buffer; training draws
 * batches from it (MSE on dE/16, Adam) with hand-written kernels.
 * Feature layout (float): badness of u, v, u^1, v^1 (/16); their rows and
 * columns (/n); the chain's 150 slot badness values (/16); zero padding.
 * ------------------------------------------------------------------------- */
typedef struct n3_mlp {
  float* params;        /* [n3_mlp_param_count()] fp32: W1[256][192] b1[256] W2[256][256] b2[256] w3[256] b3 */
  uint8_t* w2_img;      /* 131072 B: bf16 W2 in the tensor-core shared-memory layout (n3_mlp_pack) */
  uint8_t* w1a_img;     /* 8192 B: bf16 candidate columns of W1, tensor-core layout */
  uint8_t* a1_img;      /* [C][4096 B]: candidate features of each chain's 128 candidates (bf16) */
  float* badn;          /* [C][150]: chain features (badness / 16) */
  float* c1;            /* [C][256]: chain part of layer 1 (W1b x + b1) */
  int32_t* cand;        /* [C][128]: u | v << 8 | legal << 31 */
  float* pred;          /* [C][128]: predicted dE */
  uint16_t* rb_feat;    /* [capacity][12] bf16 candidate features */
  uint8_t* rb_bad;      /* [capacity][150] chain badness (clamped to 255) */
  int16_t* rb_dE;       /* [capacity] exact dE */
  int64_t rb_capacity;
  float* stats;         /* [4]: sum |pred - dE|, proposals, accepted, sum of accepted dE */
  uint64_t* counters;   /* [2]: learned steps taken (ring position, candidate stream), Adam steps taken */
  float* loss_out;      /* [1] sum of squared errors of the last training batch, or NULL */
  uint32_t* error_word; /* device error bits (8: a bounded tensor-core wait expired) */
} n3_mlp;

int n3_mlp_param_count(void);
/* Floats of training scratch needed for a batch of `batch` tuples. */
int n3_mlp_scratch_floats(int batch);
/* Rebuilds w2_img and w1a_img from params. */
int n3_mlp_pack(const n3_mlp* mlp, void* stream);
/* Draws 128 candidates per chain for the current step (Philox keyed by seed,
 * counter = step, chain, candidate), writes a1_img, badn, cand, and c1 (the
 * chain part of layer 1, one GEMM over all chains).  bad_bias (0..100) is the
 * percentage of candidates whose slot u is drawn in proportion to badness, as
 * in the reference walk (src/no_three_75/tempering.py:51-55). */
int n3_mlp_candidates(const n3_chains* chains, const n3_mlp* mlp, uint64_t seed, int bad_bias, void* stream);
/* pred[t][j] for `tiles` tiles of 128 candidates from a1_img and c1 (tcgen05). */
int n3_mlp_infer(const n3_mlp* mlp, int tiles, void* stream);
/* Samples, scores exactly, accepts and records `moves` moves per chain
 * (drawn without replacement from this step's 128 candidates, each re-checked
 * for legality on the current state; 1 is the plain learned step), then
 * advances the step counter.  temps: the ladder's L temperatures (device). */
int n3_mlp_step(const n3_chains* chains, const n3_mlp* mlp, const float* temps, uint64_t seed, int moves,
                void* stream);
/* The same step with the width of the team that works on one chain chosen by
 * the caller: threads_per_chain 32 (one warp) or 64 (two warps sharing the
 * chain's histogram); 0 takes the default (64 for several moves per step, 32
 * for one).  No counterpart in the reference.  Results do not depend on the
 * width.  A ring buffer capacity below 1 is rejected with N3_ERR_ARG. */
int n3_mlp_step_team(const n3_chains* chains, const n3_mlp* mlp, const float* temps, uint64_t seed, int moves,
                     int threads_per_chain, void* stream);
/* One Adam step on a batch drawn from the ring slots recorded so far (all
 * counters live on the device, so the call is graph-capturable); scratch
 * holds n3_mlp_scratch_floats(batch) floats, grads/adam_m/adam_v
 * n3_mlp_param_count() floats each. */
int n3_mlp_train(const n3_mlp* mlp, int n_chains, int batch, float lr, uint64_t seed, float* scratch, float* grads,
                 float* adam_m, float* adam_v, void* stream);

/* The same training step without caller-provided scratch.  No counterpart in
 * the reference.  For callers that cannot call cudaMalloc, such as a host
 * application whose own allocator takes all device memory at start-up, or a
 * plug-in whose host forbids allocations it does not make itself: the batch
 * activations and the gradient live in a static device array inside libn3.so
 * (about 4 MB, held by every GPU that loads the library until the process
 * exits), so this call allocates nothing.  batch must lie in [64, 512]; larger
 * batches are rejected with N3_ERR_RANGE.  The first call on a device looks up
 * the array's device address; make that first call before any stream capture.
 * The address is looked up again after the device's context has changed (a
 * cudaDeviceReset), so make the first call after such a reset outside any
 * capture as well.
 * All calls share the array, which keeps the last call's contents (the call
 * clears what must start at zero): calls that overlap on the GPU, from several
 * streams or threads, race on it and must be serialised by the caller. */
int n3_mlp_train_noalloc(const n3_mlp* mlp, int n_chains, int batch, float lr, uint64_t seed, float* adam_m,
                         float* adam_v, void* stream);

/* ---------------------------------------------------------------------------
 * Conflict analysis: the lines behind a score.
 * ------------------------------------------------------------------------- */

/* Every line holding three or more points of each of B point sets (m points
 * each, coordinates (row, col) in [0, N3_MAX_N), m <= 160), with each point's
 * badness.  Replaces conflicts.analyze_points (src/no_three_75/conflicts.py:36-72)
 * and its per-pair geometry.canonical_line (src/no_three_75/geometry.py:14-28).
 *   points     int16 [B][m][2]
 *   badness    int32 [B][m]: sum over lines through the point of C(k-1, 2)
 *   line_count int32 [B]: lines found, or -1 for a set with a point outside the
 *              grid, two equal points (the reference raises ValueError) or more
 *              lines than `capacity` (error bits 1, 2 and 32 of *error_word)
 *   lines      int32 [B][capacity][9]: A, B, C (the reference's canonical line:
 *              A x + B y + C = 0 over (row, col), gcd 1, A > 0 or A = 0 < B),
 *              occupancy k, then a 160-bit member mask (bit t of word w is
 *              point 32 w + t); lines in no particular order */
int n3_analyze_lines(const int16_t* points, int B, int m, int32_t* badness, int32_t* line_count,
                     int32_t* lines, int capacity, uint32_t* error_word, void* stream);

/* ---------------------------------------------------------------------------
 * Multi-point moves.
 * ------------------------------------------------------------------------- */

/* Scores after three-cycles (src/no_three_75/accelerated.py:196-276,
 * evaluate_three_cycles): candidate (u, v, w, o) moves u <- v <- w <- u (o = 0)
 * or u <- w <- v <- u (o = 1) column-wise; scores[k] = current + exact dE.
 * Candidates must be the kind search.py:38-65 generates (three rows, three
 * distinct columns, no repeated column in a row afterwards); any other gets
 * 1 << 60.  p, q int32 [n]; candidates int32 [count][4]; scores int64 [count]. */
int n3_three_cycle_scores(const int32_t* p, const int32_t* q, int n, const int32_t* candidates, int count,
                          int64_t current, int64_t* scores, void* stream);

/* Every four-cycle and double switch through slot `anchor`
 * (src/no_three_75/gpu_neighborhood.py:70-211, best_four_cycle and
 * best_double_switch), scored exactly.  best[0] / best[1] receive
 * (score << 32 | index) of the lowest-scoring legal four-cycle / double switch,
 * the index counting candidates in the reference's enumeration order (row
 * triple, layers, ordering or pairing), the first one on ties; legal[0] /
 * legal[1] the number of legal candidates.  current: E of the state.
 * best, legal: device uint64 [2] each. */
int n3_neighborhood_scan(const int32_t* p, const int32_t* q, int n, int anchor, int64_t current,
                         unsigned long long* best, unsigned long long* legal, void* stream);

/* ---------------------------------------------------------------------------
 * Line-weighted energies of breakout search (src/no_three_75/breakout.py:39-86):
 * a line (a, b, c), the points with a*row + b*col + c == 0, of weight w > 1
 * adds (w - 1) * C(occupancy, 3) to E; weights <= 1 add nothing.
 * lines int32 [n_lines][3], weights int32 [n_lines] (n_lines <= 4096).
 * ------------------------------------------------------------------------- */

/* weighted_candidate_scores (breakout.py:39-75): for the selected slot u and each
 * partner slot v, scores[v] = raw[v] + the weighted extra of the state after
 * u and v exchange columns (u to (row u, column v), v to (row v, column u)),
 * occupancies counted as the reference counts them.  raw, scores int64 [2n]
 * (raw as evaluate_two_switches returns it, sentinels included). */
int n3_weighted_switch_scores(const int32_t* p, const int32_t* q, int n, int u, const int64_t* raw,
                              const int32_t* lines, const int32_t* weights, int n_lines, int64_t* scores,
                              void* stream);

/* weighted_state_score (breakout.py:78-86) over a population: scores[b] =
 * raw[b] + sum over weighted lines of (w - 1) C(occupancy, 3).
 * p, q int32 [B][n]; raw, scores int64 [B]. */
int n3_weighted_state_scores(const int32_t* p, const int32_t* q, int B, int n, const int64_t* raw,
                             const int32_t* lines, const int32_t* weights, int n_lines, int64_t* scores,
                             void* stream);

/* ---------------------------------------------------------------------------
 * Line tables of the n x n grid (src/no_three_75/precompute.py:18-57,
 * build_geometry_tables, over src/no_three_75/cp_sat.py:109-157,
 * _multi_point_lines on the whole grid): every line with three or more grid
 * points that is neither a row nor a column, numbered as the reference numbers
 * it; members listed in row-major order (point id = row * n + column).
 * 1 <= n <= N3_MAX_N.  Built in two calls: the sizes, then the tables.
 * ------------------------------------------------------------------------- */

/* The lines whose first (row-major) member is each point.  line_at,
 * incidence_at: device int64 [n*n + 1], left as exclusive scans (the first
 * line id and the first CSR position of each point's lines); totals: HOST
 * int64 [2] = {line count, total incidences}.  Synchronises the stream. */
int n3_line_tables_count(int n, int64_t* line_at, int64_t* incidence_at, int64_t* totals, void* stream);

/* The tables of GeometryTables: offsets int64 [line_count + 1] (CSR),
 * indices int32 [incidences], pair_to_line int32 [n*n (n*n - 1) / 2] (the
 * line of each unordered pair of grid points in triangular_pair_index order,
 * precompute.py:28-33, or -1). */
int n3_line_tables_build(int n, const int64_t* line_at, const int64_t* incidence_at, int64_t line_count,
                         int64_t* offsets, int32_t* indices, int32_t* pair_to_line, void* stream);

/* score_pair_table (precompute.py:60-81) for `lists` point lists: list i holds
 * point ids ids[starts[i] .. starts[i+1]) (at most 512 points, ids distinct and
 * in [0, n*n)); scores int64 [lists] = sum over the table's lines of C(k, 3).
 * error_word (device uint32) gets bit 0 for an id out of range, bit 1 for an id
 * listed twice (the reference raises ValueError for both), bit 2 if a list's
 * lines overflow the per-warp hash (not possible within 512 points). */
int n3_lines_score_pairs(const int32_t* ids, const int64_t* starts, int lists, int n, const int32_t* pair_to_line,
                         int64_t* scores, uint32_t* error_word, void* stream);

/* score_csr (precompute.py:84-89) for `lists` point lists (any size; a point
 * listed twice counts once).  occupancy: device uint32 scratch
 * [ceil(lists / 32)][n*n]; scores int64 [lists]; error_word bit 0 for an id
 * out of [0, n*n). */
int n3_lines_score_csr(const int32_t* ids, const int64_t* starts, int lists, int n, int64_t line_count,
                       const int64_t* offsets, const int32_t* indices, uint32_t* occupancy, int64_t* scores,
                       uint32_t* error_word, void* stream);

/* ---------------------------------------------------------------------------
 * Device-resident beam search: the generation loop of
 * src/no_three_75/gpu_device_search.py:254-432 (gpu_device_beam_search) with
 * mutation, scoring, selection (including its random.Random shuffle) and
 * elite ranking all on the device, so a generation needs no host round trip.
 * ------------------------------------------------------------------------- */

/* The mutation kernel mutate_population (gpu_device_search.py:27-114, its
 * test-facing wrapper mutate_population_device :206-251): child c copies
 * parent c when c < parent_count, otherwise a parent drawn from the first
 * quality_count (160/256) or all parents, then applies 1..active_strength
 * (1 in 32: 1..max_strength) same-slot-layer column swaps, the first slot drawn
 * by parent badness with probability bad_bias/100; xorshift64* per child
 * seeded from (seed, child, generation).  Bit-identical to the reference.
 *   parent_p, parent_q int32 [parent_count][n], parent_badness int32 [parent_count][2n]
 *   child_p, child_q   int32 [population][n] */
int n3_beam_mutate(const int32_t* parent_p, const int32_t* parent_q, const int32_t* parent_badness,
                   int parent_count, int quality_count, int n, int population, int active_strength,
                   int max_strength, int bad_bias, uint64_t seed, int generation, int32_t* child_p,
                   int32_t* child_q, void* stream);

/* Canonical P/Q of B row/column 2-factors given as raw rows p[b][r], q[b][r]
 * (host pointers, int32 [B][n]; the two columns of each row in either order):
 * P is the perfect matching that augmenting paths find with the rows in order
 * and each row's columns ascending, Q the other column of each row.  Host code,
 * no GPU.  N3_ERR_ARG if a state is not a 2-factor.
 * Replaces: state.points_to_permutations (src/no_three_75/state.py:47-85) as the
 * beam searches use it on raw rows (gpu_device_search.py:178-182). */
int n3_normalize_pairs(const int32_t* p, const int32_t* q, int B, int n, int32_t* p_out, int32_t* q_out);

/* Python's random.Random(seed) (MT19937 seeded by init_by_array over the 32-bit
 * words of |seed|), used by the reference for its diversity shuffle
 * (gpu_device_search.py:280, 343).  state: device uint32[625] (624 words and
 * the position). */
int n3_py_random_seed(uint32_t* state, uint64_t seed, void* stream);
/* random.Random.shuffle(values[0..count)) with that state (count <= 65536),
 * advancing it exactly as CPython does (_randbelow by getrandbits). */
int n3_py_random_shuffle(uint32_t* state, int32_t* values, int count, void* stream);

/* The draws of random.shuffle over `count` items from the same state, without
 * applying them: steps_j[s] = the j that step s (count - 1 down to 1) swaps
 * with, steps_j[0] = 0; the state advances exactly as the shuffle's does.  The
 * beam selection resolves its window shuffle this way (one CTA; the draws of a
 * wide bit width are resolved by the whole CTA at once).  count <= 65536.
 * Replaces: the draws of rng.shuffle(diverse) (gpu_device_search.py:352). */
int n3_py_shuffle_steps(uint32_t* state, int count, int32_t* steps_j, void* stream);

#define N3_BEAM_STATUS 8 /* int64 status words, see n3_beam */

typedef struct n3_beam {
  int n, population, elite_size, energy_window, max_strength, bad_bias;
  uint64_t seed;
  int32_t* elite_p;         /* [elite_size][n] elites, ranked (rank_elites order) */
  int32_t* elite_q;         /* [elite_size][n] */
  int32_t* elite_badness;   /* [elite_size][2n] */
  int32_t* elite_scores;    /* [elite_size] */
  int32_t* child_p;         /* [population][n] this generation's children */
  int32_t* child_q;         /* [population][n] */
  int32_t* child_scores;    /* [population] */
  int32_t* pick_p;          /* [elite_size][n] selected children before ranking */
  int32_t* pick_q;          /* [elite_size][n] */
  int32_t* pick_badness;    /* [elite_size][2n] */
  int32_t* pick_scores;     /* [elite_size] */
  int32_t* selected;        /* [elite_size] child indices */
  uint32_t* rng;            /* [625] random.Random(seed) state */
  int64_t* status;          /* [N3_BEAM_STATUS]: elite count, best E, best max badness, best sum of
                               squared badness, last improvement, generations completed,
                               this generation's best E, improved (0/1) */
  int32_t* best_p;          /* [n] best state so far (raw P/Q rows) */
  int32_t* best_q;          /* [n] */
  int32_t* history;         /* [history_len][2] per generation: its best E, best E so far (or NULL) */
  int history_len;
  int32_t* child_parent;    /* [population] the elite each child copies */
  int32_t* child_moves;     /* [population][max_strength] its swaps, u | v << 8, in order */
  int32_t* child_nmoves;    /* [population] how many */
  int32_t* child_badness;   /* [population][2n] badness of each child */
  uint32_t* error_word;     /* device error bits (16: a maintained badness failed its re-check), or NULL */
} n3_beam;

/* Set-up: elite rows [0, base_count) hold the initial state and any supplied
 * elites (base_count <= elite_size); scores and ranks them, records the best
 * and seeds the shuffle RNG with the search seed (gpu_device_search.py:279-313). */
int n3_beam_init(const n3_beam* beam, int base_count, void* stream);
/* One generation (gpu_device_search.py:315-411): mutate the elites into
 * population children, score them (each child's E and badness from its parent's
 * by the exact delta of each of its swaps, the reference rescoring every child
 * in full), keep the best quarter plus a shuffled pick
 * of the children within energy_window of the best, fill from the score order,
 * rank by (E, max badness, sum of squared badness) and update the best.  Does
 * nothing once a generation has reached E = 0.  population <= 65536,
 * elite_size <= 2048. */
int n3_beam_generation(const n3_beam* beam, int generation, void* stream);

/* Device clock (%globaltimer, ns) written to *out (device int64) in stream
 * order; used to time a run to its first target hit on the device. */
int n3_device_clock_ns(int64_t* out, void* stream);

/* ---------------------------------------------------------------------------
 * CUDA graphs (no reference counterpart: the reference launches every epoch
 * from Python, src/no_three_75/tempering.py:275-278).  Capture the launches
 * made on `stream` between n3_graph_begin and n3_graph_end (thread-local
 * capture mode), then replay them with n3_graph_launch.
 * ------------------------------------------------------------------------- */
int n3_graph_begin(void* stream);
int n3_graph_end(void* stream, void** graph_exec);
int n3_graph_launch(void* graph_exec, void* stream);
int n3_graph_destroy(void* graph_exec);

/* ---------------------------------------------------------------------------
 * Measurement helper (no reference counterpart).
 * ------------------------------------------------------------------------- */

/* Runs the scorer's determinant test expression on register operands only
 * (no memory traffic): blocks x 256 threads x iters x 16 triple tests.  Its
 * event-timed rate is the integer-pipe ceiling that bench.py reports the
 * scorer's rate against.  scratch2: device uint64[2]. */
int n3_calibrate_det_ceiling(int blocks, int iters, unsigned long long* scratch2, void* stream);

/* Throughput of one integer pipe on its own: blocks x 256 threads x iters x 8
 * dependent-chain operations, kind 0 an integer multiply-add (the FMA pipe,
 * which the scorer's products use), kind 1 a three-input logic operation (the
 * ALU pipe, which its compares use).  Event-timed, these are the pipe ceilings
 * bench.py states the scorer's roofline against.  scratch2: device uint64[2]. */
int n3_calibrate_int_pipe(int kind, int blocks, int iters, unsigned long long* scratch2, void* stream);

/* Random 4-byte gathers from `table` (int32 [entries], sized to stay in L2):
 * blocks x 256 threads x iters loads at xorshift-drawn indices.  Event-timed,
 * the rate is the ceiling bench.py states the pair-table scorer's gathers
 * against.  scratch2: device uint64[2]. */
int n3_calibrate_l2_gather(const int32_t* table, int64_t entries, int blocks, int iters,
                           unsigned long long* scratch2, void* stream);

/* Makes one bounded device wait expire, safely: an mbarrier that nothing
 * arrives on is waited for at most `tries` times (1 .. 2^20) with the wait
 * the tensor-core pipeline uses, which then ORs error bit 8 (a bounded wait
 * gave up) into *error_word and returns.  Lets callers and tests check the
 * expiry path without hanging or faulting the GPU.  No reference counterpart. */
int n3_check_bounded_wait(uint32_t tries, uint32_t* error_word, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* N3_H_ */
