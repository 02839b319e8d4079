// kernel_ids.h -- kernel classes for per-kernel statistics (device time, launches, NCC evaluations).
#pragma once

enum KernelId {
  KID_INIT_STATE = 0,
  KID_GEN_EDGE_INFORM,
  KID_FIND_NEAREST,
  KID_GEN_NEIGHBOURS,
  KID_NEIGHBOUR_UPDATE,
  KID_RANDOM_INIT,
  KID_STRONG_UPDATE,
  KID_RANSAC,
  KID_WEAK_PREPARE,
  KID_WEAK_EVAL,
  KID_WEAK_DECIDE,
  KID_WEAK_FINISH,
  KID_DEPTH_NORMAL,
  KID_FILTER,
  KID_DEPTH_TO_WEAK,
  KID_LOCAL_REFINE,
  KID_PAD_IMAGE,
  KID_NCC_QUERY,
  KID_FUSE_ENTRIES,
  KID_FUSE_ROUNDS,
  KID_FUSE_EMIT,
  KID_FUSE_TAT,
  KID_EDGE_MAP,
  KID_EDGE_LABELS,
  KID_SCENE_MISC,
  KID_COUNT
};

static const char *const kKernelNames[KID_COUNT] = {
    "k_init_state",    "k_gen_edge_inform", "k_find_nearest_strong", "k_gen_neighbours", "k_neighbour_update",
    "k_random_init",   "k_strong_update",   "k_ransac_fit_plane",    "k_weak_prepare",   "k_weak_eval",
    "k_weak_decide",   "k_weak_finish",     "k_get_depth_normal",
    "k_filter_strong", "k_depth_to_weak",   "k_local_refine",        "k_pad_image",      "k_ncc_queries",
    "k_fuse_entries",  "k_fuse_rounds",      "k_fuse_emit",           "k_fuse_tat",       "k_edge_map",
    "k_edge_labels",   "k_scene_misc"};
