"""Streaming host-memory batches through a transform with copies overlapped.

`HostPipeline` runs `step(device_in, device_out)` over a sequence of pinned
host input batches, writing each result into the matching pinned host output
batch.  Three CUDA streams and two device buffers per side overlap, for
consecutive batches i - 1, i, i + 1, the download of i - 1, the transform of
i and the upload of i + 1; each batch still makes its full host -> device
and device -> host trip.  Events order the reuse of every device buffer.
This is the streaming counterpart of the reference's `wavemoth_execute`
(src/wavemoth.c:1271-1283), which runs one bound host batch at a time.
"""
import torch


class HostPipeline:
    def __init__(self, in_shape, in_dtype, out_shape, out_dtype, step, device="cuda"):
        self.step = step
        self.d_in = [torch.empty(in_shape, dtype=in_dtype, device=device) for _ in range(2)]
        self.d_out = [torch.empty(out_shape, dtype=out_dtype, device=device) for _ in range(2)]
        self.s_in = torch.cuda.Stream(device=device)
        self.s_run = torch.cuda.Stream(device=device)
        self.s_out = torch.cuda.Stream(device=device)
        self.in_ready = [torch.cuda.Event() for _ in range(2)]
        self.in_free = [torch.cuda.Event() for _ in range(2)]
        self.out_ready = [torch.cuda.Event() for _ in range(2)]
        self.out_free = [torch.cuda.Event() for _ in range(2)]

    def run(self, host_inputs, host_outputs):
        """Processes every (host_inputs[i] -> host_outputs[i]); returns after
        enqueueing (synchronise the device, or the current stream, which is
        made to wait for the last download, before reading the outputs)."""
        if len(host_inputs) != len(host_outputs):
            raise ValueError("inputs and outputs differ in length")
        cur = torch.cuda.current_stream()
        for s in (self.s_in, self.s_run, self.s_out):
            s.wait_stream(cur)
        for i, (hi, ho) in enumerate(zip(host_inputs, host_outputs)):
            b = i & 1
            with torch.cuda.stream(self.s_in):
                if i >= 2:
                    self.s_in.wait_event(self.in_free[b])
                self.d_in[b].copy_(hi, non_blocking=True)
                self.in_ready[b].record(self.s_in)
            with torch.cuda.stream(self.s_run):
                self.s_run.wait_event(self.in_ready[b])
                if i >= 2:
                    self.s_run.wait_event(self.out_free[b])
                self.step(self.d_in[b], self.d_out[b])
                self.in_free[b].record(self.s_run)
                self.out_ready[b].record(self.s_run)
            with torch.cuda.stream(self.s_out):
                self.s_out.wait_event(self.out_ready[b])
                ho.copy_(self.d_out[b], non_blocking=True)
                self.out_free[b].record(self.s_out)
        cur.wait_stream(self.s_out)
