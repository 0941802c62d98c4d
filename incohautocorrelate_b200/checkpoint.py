"""Checkpoint and resume of a long correlation run.

The reference has none: a run over an event list is one process from start to
end (IAC/RunIAC.cpp:524-550), and only its final products are written.  Here the
state of a run is exact and small: the uint64 half mesh binned so far and the
index of the next frame.  Mesh values are integer sums, which commute, so a run
that stops after any batch and resumes from its last checkpoint ends with the
very mesh an uninterrupted run gives, bit for bit.

    run = MeshRun(ctx, params, S)                # or MeshRun.resume(ctx, path)
    run.bin_frames(photons, offsets, rot, batch=4096, checkpoint=path, every=8)
    full = run.full_mesh()                       # folded, uint64[S^3]

A checkpoint is one .npz file, written to a temporary name and renamed, so a
crash while saving leaves the previous checkpoint intact.  It records which
event list was being binned (frame count and a digest of the frame offsets and
rotations), and a resumed run refuses to continue on another list, which would
silently mix two runs into one mesh at the saved cursor.
"""
from __future__ import annotations

import hashlib
import os

import numpy as np

_FORMAT = 2


def event_list_digest(offsets, rot) -> str:
    """Identity of an event list: its frame count and a SHA-256 of its frame
    offsets and rotation matrices."""
    off = np.ascontiguousarray(offsets, np.uint64)
    h = hashlib.sha256()
    h.update(np.int64(len(off) - 1).tobytes())
    h.update(off.tobytes())
    h.update(np.ascontiguousarray(rot, np.float32).tobytes())
    return h.hexdigest()


class MeshRun:
    """Frames binned into one device half mesh, in batches, from a cursor."""

    def __init__(self, ctx, params, S: int, half=None, cursor: int = 0, events: str | None = None):
        import torch

        from . import capi
        self.ctx, self.params, self.S = ctx, params, int(S)
        words = capi.half_mesh_words(self.S)
        if half is None:
            self.half = torch.zeros(words, dtype=torch.int64, device="cuda")
        else:
            h = np.ascontiguousarray(half, np.uint64).view(np.int64)
            if h.size != words:
                raise ValueError(f"checkpoint half mesh has {h.size} words, mesh {self.S} needs {words}")
            self.half = torch.from_numpy(h).cuda()
        self.cursor = int(cursor)
        self.events = events  # digest of the event list being binned (set by the first bin_frames)

    # -- state ---------------------------------------------------------------
    def _key(self) -> np.ndarray:
        p = self.params
        s = p.shape
        return np.array([s.k_a, s.k_b, s.k_c, s.size_ab, s.size_c, s.voxel_per_dq, p.interp_first,
                         p.interp_second, p.double_map], np.int64)

    def save(self, path: str):
        """Write the half mesh, the cursor and what the mesh depends on."""
        self.ctx.check()
        tmp = path + ".tmp.npz"
        np.savez(tmp, format=_FORMAT, half=self.half.cpu().numpy().view(np.uint64), cursor=self.cursor,
                 key=self._key(), max_q=np.float32(self.params.shape.max_q),
                 multiplicator=np.float64(self.params.multiplicator), events=self.events or "")
        os.replace(tmp, path)

    @classmethod
    def resume(cls, ctx, params, S: int, path: str) -> "MeshRun":
        """Continue the run saved at `path`; the parameters must be the saved ones."""
        with np.load(path) as z:
            if int(z["format"]) != _FORMAT:
                raise ValueError(f"{path}: checkpoint format {int(z['format'])}, expected {_FORMAT}")
            run = cls(ctx, params, S, half=z["half"], cursor=int(z["cursor"]), events=str(z["events"]) or None)
            if not (np.array_equal(z["key"], run._key()) and float(z["max_q"]) == float(np.float32(params.shape.max_q))
                    and float(z["multiplicator"]) == float(params.multiplicator)):
                raise ValueError(f"{path}: saved with other mesh or binning parameters")
        return run

    # -- work ----------------------------------------------------------------
    def bin_frames(self, photons, offsets, rot, batch: int = 4096, checkpoint: str | None = None,
                   every: int = 1, stop_after: int | None = None) -> int:
        """Bin frames cursor .. end in batches of `batch` frames, saving to
        `checkpoint` after every `every` batches and at the end.  `stop_after`
        ends the call after that many batches (a run cut short).  Returns the
        cursor."""
        import torch
        off = np.asarray(offsets, np.uint64)
        nframes = len(off) - 1
        digest = event_list_digest(off, rot)
        if self.events is None:
            self.events = digest
        elif self.events != digest:
            raise ValueError("the run was binning another event list (frame count, offsets or rotations differ); "
                             "resuming it on this one would mix two runs into one mesh")
        done = 0
        while self.cursor < nframes:
            f0, f1 = self.cursor, min(nframes, self.cursor + int(batch))
            p0, p1 = int(off[f0]), int(off[f1])
            ph = np.ascontiguousarray(photons[p0:p1] if p1 > p0 else np.zeros((1, 4), np.float32), np.float32)
            d_ph = torch.from_numpy(ph).cuda()
            d_off = torch.from_numpy((off[f0:f1 + 1] - off[f0]).view(np.int64).copy()).cuda()
            d_rot = torch.from_numpy(np.ascontiguousarray(rot[f0:f1], np.float32)).cuda()
            self.ctx.sparse_ac_batch(d_ph, d_off, d_rot, f1 - f0, self.params, self.half)
            self.cursor = f1
            done += 1
            if checkpoint and (done % max(1, int(every)) == 0 or self.cursor == nframes):
                self.save(checkpoint)
            if stop_after is not None and done >= stop_after:
                break
        return self.cursor

    def full_mesh(self) -> np.ndarray:
        """The folded mesh of every frame binned so far (uint64[S^3])."""
        import torch

        from . import capi
        full = torch.zeros(capi.full_mesh_words(self.S), dtype=torch.int64, device="cuda")
        self.ctx.sparse_fold(self.half, self.S, full)
        self.ctx.check()
        return full.cpu().numpy().view(np.uint64)
