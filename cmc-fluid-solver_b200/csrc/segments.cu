// Segment builder: turns the node mask into per-direction segment descriptors.
//
// Restates Grid3D::GenerateListSegments (Grid3D.cpp:47-127) with nblockZ = 1 as
// two data-parallel passes, one thread per line:
//   pass 1 (segment_scan):  segments per line, first/last segment node, longest
//                           segment and node count per line;
//   (host: exclusive scan of the per-line counts = each line's output offset)
//   pass 2 (segment_write): the descriptors, written at the line's offset.
// Lines are numbered in the order the reference visits them, so the concatenated
// output equals the reference's list entry for entry.  Along a line, a segment
// opens at the cell before the first IN cell of a run (the predecessor may be any
// non-IN cell, or cell 0) and closes at the first non-IN cell after the run; a run
// that reaches the last cell is dropped, as in the reference.
//
// For X and Y the line number's fastest index is k, so neighbouring threads read
// neighbouring bytes; Z lines are contiguous per thread (setup-only cost).
#include "adi_internal.cuh"

namespace adi {

__global__ void segment_scan_kernel(int dir, LineGeom g, const uint8_t *__restrict__ code, int *line_count,
                                    int *line_lo, int *line_hi, int *line_maxlen, long long *line_nodes)
{
    int line = blockIdx.x * blockDim.x + threadIdx.x;
    if (line >= g.nlines) return;
    const long long base = line_base(dir, g, line);
    int count = 0, lo = -1, hi = -1, maxlen = 0, state = 0, start = 0;
    long long nodes = 0;
    for (int q = 0; q + 1 < g.len; q++) {
        bool in = code_is_in(code[base + (long long)(q + 1) * g.stride]);
        if (in) {
            if (!state) start = q;
            state = 1;
        } else if (state) {
            int size = q + 1 - start + 1;
            if (count == 0) lo = start;
            hi = q + 1;
            count++;
            nodes += size;
            maxlen = size > maxlen ? size : maxlen;
            state = 0;
        }
    }
    line_count[line] = count;
    line_lo[line] = lo;
    line_hi[line] = hi;
    line_maxlen[line] = maxlen;
    line_nodes[line] = nodes;
}

__global__ void segment_write_kernel(int dir, LineGeom g, const uint8_t *__restrict__ code,
                                     const long long *__restrict__ line_offset, int32_t *out7)
{
    int line = blockIdx.x * blockDim.x + threadIdx.x;
    if (line >= g.nlines) return;
    const long long base = line_base(dir, g, line);
    int p[3];
    if (dir == 0) { p[0] = 0; p[1] = line / g.nz; p[2] = line % g.nz; }
    else if (dir == 1) { p[0] = line / g.nz; p[1] = 0; p[2] = line % g.nz; }
    else { p[0] = line / g.ny; p[1] = line % g.ny; p[2] = 0; }
    long long o = line_offset[line];
    int state = 0, start = 0;
    for (int q = 0; q + 1 < g.len; q++) {
        bool in = code_is_in(code[base + (long long)(q + 1) * g.stride]);
        if (in) {
            if (!state) start = q;
            state = 1;
        } else if (state) {
            int32_t *w = out7 + 7 * o;
            w[0] = p[0]; w[1] = p[1]; w[2] = p[2];
            w[dir] = start;
            w[3] = p[0]; w[4] = p[1]; w[5] = p[2];
            w[3 + dir] = q + 1;
            w[6] = q + 1 - start + 1;
            o++;
            state = 0;
        }
    }
}

cudaError_t launch_segment_scan(int dir, int nx, int ny, int nz, const uint8_t *code, int *line_count,
                                int *line_lo, int *line_hi, int *line_maxlen, long long *line_nodes,
                                cudaStream_t s)
{
    LineGeom g = line_geom(dir, nx, ny, nz);
    int threads = 128, blocks = (g.nlines + threads - 1) / threads;
    segment_scan_kernel<<<blocks, threads, 0, s>>>(dir, g, code, line_count, line_lo, line_hi, line_maxlen,
                                                     line_nodes);
    return cudaGetLastError();
}

cudaError_t launch_segment_write(int dir, int nx, int ny, int nz, const uint8_t *code,
                                 const long long *line_offset, int32_t *out7, cudaStream_t s)
{
    LineGeom g = line_geom(dir, nx, ny, nz);
    int threads = 128, blocks = (g.nlines + threads - 1) / threads;
    segment_write_kernel<<<blocks, threads, 0, s>>>(dir, g, code, line_offset, out7);
    return cudaGetLastError();
}

} // namespace adi
