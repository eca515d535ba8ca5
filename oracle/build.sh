#!/bin/sh
# Builds the test oracle (TEST INFRASTRUCTURE ONLY): liboracle.so always, and,
# where the reference checkout is present on this machine, the reference's own
# C compiled from its sources into oracle/_ref (see Makefile). The checkout is
# read where it lies: $BC250_REFERENCE if set, else the read-only mount of the
# build container. On a machine without it (the GPU box), make keeps the
# prebuilt oracle/_ref that travelled with the tree.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT_REF=${BC250_REFERENCE:-/root/reference}
if [ -f "$ROOT_REF/approach1-compute-encoder/src/h264_deblock.c" ]; then
    exec make -s -C "$HERE" REF="$ROOT_REF/approach1-compute-encoder" "$@"
fi
exec make -s -C "$HERE" "$@"
