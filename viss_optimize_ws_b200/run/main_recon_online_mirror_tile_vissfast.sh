#!/usr/bin/env bash
# Parameter script for the B200 drop-in of main_recon_online_mirror_tile_vissfast
# (mirrored half grid, tile-cone culling, occ_mode=2 representatives).  Same
# flags as the upstream script; values can be overridden from the environment.
# Prints start / end time, elapsed time and the exit code like the upstream one.
set -u
HERE="$(cd "$(dirname "$0")" && pwd)"
EXE="${EXE:-$HERE/../bin/main_recon_online_mirror_tile_vissfast}"

BTAG="${BTAG:-10M}"
NSIDE="${NSIDE:-4096}"
DAY_START="${DAY_START:-1}"
DAY_COUNT="${DAY_COUNT:-1}"
SEGS="${SEGS:-10}"
SKY_DIR="${SKY_DIR:-../earth_10Mhz}"
OUT_DIR="${OUT_DIR:-../out10M_vissfast/}"
GPUS="${GPUS:-0}"

echo "========================================"
echo "start: $(date '+%Y-%m-%d %H:%M:%S')"
echo "========================================"
T0=$(date +%s)

"$EXE" \
  --btag="$BTAG" \
  --nside="$NSIDE" \
  --day_start="$DAY_START" \
  --day_count="$DAY_COUNT" \
  --segs="$SEGS" \
  --blockage=1 \
  --occ_mode=2 \
  --sky_dir="$SKY_DIR" \
  --out_dir="$OUT_DIR" \
  --gpus="$GPUS" \
  --gen_gpu_index=0 \
  --B_mode=bin \
  --C_mode=bin \
  --orbit_seed=42 \
  "$@"
RC=$?

T=$(( $(date +%s) - T0 ))
echo ""
echo "========================================"
echo "end: $(date '+%Y-%m-%d %H:%M:%S')"
printf 'elapsed: %dh %dm %ds\n' $((T / 3600)) $(((T % 3600) / 60)) $((T % 60))
echo "exit code: ${RC}"
echo "========================================"
exit ${RC}
