#!/usr/bin/env bash
# Parameter script for the B200 drop-in of main_recon_online (root variant).
# The flag set is the upstream one (main_recon_online.sh); the binary accepts it
# unchanged.  Every value can be overridden from the environment, e.g.
#   BTAG=1M NSIDE=512 SKY_DIR=./earth_1Mhz ./main_recon_online.sh
# --gpus / --gen_gpu_index only select the device: the build runs on one GPU.
set -u
HERE="$(cd "$(dirname "$0")" && pwd)"
EXE="${EXE:-$HERE/../bin/main_recon_online}"

BTAG="${BTAG:-10M}"
NSIDE="${NSIDE:-4096}"
DAY="${DAY:-1}"
SEGS="${SEGS:-10}"
SKY_DIR="${SKY_DIR:-./earth_10Mhz}"
OUT_DIR="${OUT_DIR:-./out10M_online/}"
GPUS="${GPUS:-0}"
B_MODE="${B_MODE:-txt}"

"$EXE" \
  --btag="$BTAG" \
  --nside="$NSIDE" \
  --day="$DAY" \
  --segs="$SEGS" \
  --blockage=1 \
  --occ_mode=2 \
  --sky_dir="$SKY_DIR" \
  --out_dir="$OUT_DIR" \
  --gpus="$GPUS" \
  --gen_gpu_index=0 \
  --B_mode="$B_MODE" \
  --orbit_seed=42 \
  --write_viss=1 \
  --write_baseline_txt=1 \
  "$@"
