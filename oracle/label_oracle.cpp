// label_oracle.cpp -- CPU restatement of EdgeSegment's label map (DPE.cpp:136-291, mode 1 without
// Canny) as GetProblemEdges requests it (main.cpp:199-214), with its parts:
//   Connect (DPE.cpp:27-134), Roberts (DPE.cpp:9-25), and the OpenCV calls EdgeSegment makes:
//   cv::resize INTER_LINEAR on 8-bit images, cv::threshold, cv::HoughLinesP and cv::line.
//
// TEST INFRASTRUCTURE ONLY: the checker for the device label maps and for the host
// preprocessing.  Connect is a literal restatement of the reference loop: provisional labels in
// raster order, a join of two different labels recorded as connection[larger] = smaller
// (overwriting an earlier join of the same label, which the reference then loses), chain ends as
// final labels, renumbered in increasing order.
//
// OpenCV is a third-party dependency absent from the reference tree (OpenCV 4.x; 4.13.0 in this
// image).  Its calls are restated from their published algorithms in OpenCV's integer forms:
//   - resize, 8-bit INTER_LINEAR: source coordinate (d + 0.5) * scale - 0.5 in float; horizontal
//     weights clamped at the borders, vertical weights not (only the source row is clamped);
//     weights rounded to 11 bits; horizontal sums in int, the vertical pass in OpenCV's 16-bit
//     form ((b0 * (r0 >> 4)) >> 16) + ((b1 * (r1 >> 4)) >> 16), + 2 >> 2;
//   - HoughLinesP: the progressive probabilistic Hough transform (Matas, Galambos, Kittler, CVIU
//     2000) with OpenCV's multiply-with-carry generator (state * 4164903690 + carry, seeded with
//     all ones), a float trigonometric table, accumulator votes rounded half to even, and the
//     16.16 fixed-point walk that extracts the segment and withdraws its votes;
//   - line (thickness 1, 8-connected): the Bresenham iterator from the left end.
// PINNED against the dependency itself: tests/test_labels.py compares every part and the whole
// map with the host preprocessing, which calls cv2 as the reference calls OpenCV, bit for bit.
// Roberts and Connect are the reference's own functions: tests/test_ref_oracle.py pins this
// Connect and the host preprocessing's Roberts to them, compiled for the CPU (oracle/_ref).
#include <cmath>
#include <cstdint>
#include <vector>

extern "C" int oracle_connect(const uint8_t *img, int cols, int rows, int32_t *labels, int32_t *counts,
                              int counts_capacity, int *num_labels) {
  if (!img || !labels || cols < 1 || rows < 1) return 1;
  std::vector<int> lab((size_t)rows * cols, 0);
  std::vector<int> connection(1, 0);
  int cnt = 1;
  for (int y = 0; y < rows; ++y)
    for (int x = 0; x < cols; ++x) {
      const size_t p = (size_t)y * cols + x;
      if (img[p] == 255) {
        lab[p] = 0;
        continue;
      }
      const bool left = x > 0 && img[p] == 0 && img[p - 1] == 0;
      const bool up = y > 0 && img[p] == 0 && img[p - cols] == 0;
      if (left) lab[p] = lab[p - 1];
      if (up) lab[p] = lab[p - cols];
      if (!left && !up) {
        lab[p] = cnt;
        connection.push_back(cnt);
        cnt++;
      } else if (left && up) {
        const int l = lab[p - 1], u = lab[p - cols];
        if (l > u) {
          connection[l] = u;
          lab[p] = lab[p - cols];
        } else if (l < u) {
          connection[u] = l;
          lab[p] = lab[p - 1];
        }
      }
    }
  for (size_t i = 1; i < connection.size(); ++i) {
    int cur = connection[i], pre = connection[cur];
    while (pre != cur) {
      cur = pre;
      pre = connection[pre];
    }
    connection[i] = cur;
  }
  int label_num = 1;
  std::vector<int> mapping(connection.size(), 0);
  for (size_t i = 1; i < connection.size(); ++i)
    if (connection[i] == (int)i) mapping[i] = label_num++;
  for (size_t i = 1; i < connection.size(); ++i) connection[i] = mapping[connection[i]];
  for (int k = 0; k < counts_capacity && counts; ++k) counts[k] = 0;
  for (size_t p = 0; p < (size_t)rows * cols; ++p) {
    const int l = connection[lab[p]];
    labels[p] = l;
    if (counts && l < counts_capacity) counts[l]++;
  }
  if (num_labels) *num_labels = label_num;
  return label_num > counts_capacity ? 2 : 0;
}

namespace {

// cv::resize, 8-bit single channel, INTER_LINEAR (see the header for the arithmetic).
void resize_u8(const uint8_t *src, int sw, int sh, uint8_t *dst, int dw, int dh) {
  const double sx_scale = 1.0 / ((double)dw / sw), sy_scale = 1.0 / ((double)dh / sh);
  std::vector<int> xo(dw), xa0(dw), xa1(dw);
  for (int d = 0; d < dw; ++d) {
    float fx = (float)((d + 0.5) * sx_scale - 0.5);
    int sx = (int)std::floor(fx);
    fx -= (float)sx;
    if (sx < 0) { fx = 0.f; sx = 0; }
    if (sx >= sw - 1) { fx = 0.f; sx = sw - 1; }
    xo[d] = sx;
    xa0[d] = (int)std::nearbyint((1.f - fx) * 2048.f);
    xa1[d] = (int)std::nearbyint(fx * 2048.f);
  }
  std::vector<int> r0(dw), r1(dw);
  for (int d = 0; d < dh; ++d) {
    float fy = (float)((d + 0.5) * sy_scale - 0.5);
    const int sy = (int)std::floor(fy);
    fy -= (float)sy;
    const int b0 = (int)std::nearbyint((1.f - fy) * 2048.f), b1 = (int)std::nearbyint(fy * 2048.f);
    const int y0 = sy < 0 ? 0 : sy > sh - 1 ? sh - 1 : sy;
    const int y1 = sy + 1 < 0 ? 0 : sy + 1 > sh - 1 ? sh - 1 : sy + 1;
    for (int x = 0; x < dw; ++x) {
      const int xa = xo[x], xb = xo[x] + 1 < sw ? xo[x] + 1 : sw - 1;
      r0[x] = src[(size_t)y0 * sw + xa] * xa0[x] + src[(size_t)y0 * sw + xb] * xa1[x];
      r1[x] = src[(size_t)y1 * sw + xa] * xa0[x] + src[(size_t)y1 * sw + xb] * xa1[x];
    }
    for (int x = 0; x < dw; ++x) {
      const int v = (((b0 * (r0[x] >> 4)) >> 16) + ((b1 * (r1[x] >> 4)) >> 16) + 2) >> 2;
      dst[(size_t)d * dw + x] = (uint8_t)(v < 0 ? 0 : v > 255 ? 255 : v);
    }
  }
}

// Roberts (DPE.cpp:9-25): (uchar)sqrt(int), i.e. the truncated root's low byte.
void roberts(const uint8_t *s, int cols, int rows, uint8_t *d) {
  for (int i = 0; i < rows; ++i)
    for (int j = 0; j < cols; ++j) {
      int t1, t2;
      if (i > 0 && i < rows - 1 && j > 0 && j < cols - 1) {
        t1 = s[(size_t)i * cols + j] - s[(size_t)(i + 1) * cols + j + 1];
        t2 = s[(size_t)(i + 1) * cols + j] - s[(size_t)i * cols + j + 1];
      } else {
        t1 = t2 = 50;
      }
      d[(size_t)i * cols + j] = (uint8_t)(int)std::sqrt((double)(t1 * t1 + t2 * t2));
    }
}

struct CvRng {
  uint64_t state;
  explicit CvRng(uint64_t s) : state(s ? s : 0xffffffffu) {}
  unsigned next() {
    state = (uint64_t)(unsigned)state * 4164903690u + (unsigned)(state >> 32);
    return (unsigned)state;
  }
  int uniform(int a, int b) { return a == b ? a : (int)(next() % (unsigned)(b - a) + a); }
};

struct Seg { int x0, y0, x1, y1; };

// cv::HoughLinesP(image, lines, rho = 1, theta = CV_PI / 180, threshold, minLineLength, maxLineGap)
void hough_lines_p(const uint8_t *image, int width, int height, int threshold, int line_length, int line_gap,
                   std::vector<Seg> &lines) {
  const float rho = 1.0f, theta = (float)(3.14159265358979323846 / 180.0);
  const float irho = 1 / rho;
  int numangle = (int)std::floor((3.14159265358979323846 - 0.0) / theta) + 1;
  if (numangle > 1 && std::fabs(3.14159265358979323846 - (numangle - 1) * (double)theta) < theta / 2) --numangle;
  const int numrho = (int)std::nearbyint(((width + height) * 2 + 1) / rho);
  std::vector<int> accum((size_t)numangle * numrho, 0);
  std::vector<float> tab(2 * numangle);
  for (int n = 0; n < numangle; ++n) {
    tab[2 * n] = (float)(std::cos((double)n * theta) * irho);
    tab[2 * n + 1] = (float)(std::sin((double)n * theta) * irho);
  }
  std::vector<uint8_t> mask((size_t)width * height);
  std::vector<int> nz;  // (y << 16 | x) is not needed: store x, y pairs
  for (int y = 0; y < height; ++y)
    for (int x = 0; x < width; ++x) {
      const bool on = image[(size_t)y * width + x] != 0;
      mask[(size_t)y * width + x] = on ? 1 : 0;
      if (on) { nz.push_back(x); nz.push_back(y); }
    }
  CvRng rng(~(uint64_t)0);
  const int shift = 16;
  auto vote = [&](int x, int y, int delta, int *best_val, int *best_n) {
    for (int n = 0; n < numangle; ++n) {
      int r = (int)std::nearbyint((float)x * tab[2 * n] + (float)y * tab[2 * n + 1]);
      r += (numrho - 1) / 2;
      int &a = accum[(size_t)n * numrho + r];
      a += delta;
      if (best_val && *best_val < a) { *best_val = a; *best_n = n; }
    }
  };
  for (int count = (int)nz.size() / 2; count > 0; count--) {
    const int idx = rng.uniform(0, count);
    const int j = nz[2 * idx], i = nz[2 * idx + 1];
    nz[2 * idx] = nz[2 * (count - 1)];
    nz[2 * idx + 1] = nz[2 * (count - 1) + 1];
    if (!mask[(size_t)i * width + j]) continue;
    int max_val = threshold - 1, max_n = 0;
    vote(j, i, 1, &max_val, &max_n);
    if (max_val < threshold) continue;
    const float a = -tab[2 * max_n + 1], b = tab[2 * max_n];
    int x0 = j, y0 = i, dx0, dy0;
    bool xflag;
    if (std::fabs(a) > std::fabs(b)) {
      xflag = true;
      dx0 = a > 0 ? 1 : -1;
      dy0 = (int)std::nearbyint(b * (1 << shift) / std::fabs(a));
      y0 = (y0 << shift) + (1 << (shift - 1));
    } else {
      xflag = false;
      dy0 = b > 0 ? 1 : -1;
      dx0 = (int)std::nearbyint(a * (1 << shift) / std::fabs(b));
      x0 = (x0 << shift) + (1 << (shift - 1));
    }
    int end[2][2] = {{0, 0}, {0, 0}};
    for (int k = 0; k < 2; ++k) {
      int gap = 0, x = x0, y = y0, dx = k ? -dx0 : dx0, dy = k ? -dy0 : dy0;
      for (;; x += dx, y += dy) {
        const int j1 = xflag ? x : x >> shift, i1 = xflag ? y >> shift : y;
        if (j1 < 0 || j1 >= width || i1 < 0 || i1 >= height) break;
        if (mask[(size_t)i1 * width + j1]) {
          gap = 0;
          end[k][0] = j1;
          end[k][1] = i1;
        } else if (++gap > line_gap) {
          break;
        }
      }
    }
    const bool good = std::abs(end[1][0] - end[0][0]) >= line_length || std::abs(end[1][1] - end[0][1]) >= line_length;
    for (int k = 0; k < 2; ++k) {
      int x = x0, y = y0, dx = k ? -dx0 : dx0, dy = k ? -dy0 : dy0;
      for (;; x += dx, y += dy) {
        const int j1 = xflag ? x : x >> shift, i1 = xflag ? y >> shift : y;
        uint8_t &m = mask[(size_t)i1 * width + j1];
        if (m) {
          if (good) vote(j1, i1, -1, nullptr, nullptr);
          m = 0;
        }
        if (i1 == end[k][1] && j1 == end[k][0]) break;
      }
    }
    if (good) lines.push_back(Seg{end[0][0], end[0][1], end[1][0], end[1][1]});
  }
}

// cv::line(img, p1, p2, 255, 1): 8-connected Bresenham from the left end (points inside).
void draw_line(uint8_t *img, int width, int x1, int y1, int x2, int y2) {
  int dx = x2 - x1, dy = y2 - y1;
  if (dx < 0) { std::swap(x1, x2); std::swap(y1, y2); dx = -dx; dy = -dy; }
  long step_y = width, step_x = 1;
  if (dy < 0) { dy = -dy; step_y = -step_y; }
  if (dy > dx) { std::swap(dx, dy); std::swap(step_x, step_y); }
  int err = dx - (dy + dy);
  const int plus_delta = dx + dx, minus_delta = -(dy + dy);
  long p = (long)y1 * width + x1;
  for (int c = 0; c <= dx; ++c) {
    img[p] = 255;
    const bool m = err < 0;
    err += minus_delta + (m ? plus_delta : 0);
    p += step_x + (m ? step_y : 0);
  }
}

void border_rule(uint8_t *d, int cols, int rows) {
  for (int y = 0; y < rows; ++y) {
    if (d[(size_t)y * cols + 1] == 0) d[(size_t)y * cols] = 0;
    if (d[(size_t)y * cols + cols - 2] == 0) d[(size_t)y * cols + cols - 1] = 0;
  }
  for (int x = 0; x < cols; ++x) {
    if (d[(size_t)cols + x] == 0) d[x] = 0;
    if (d[(size_t)(rows - 2) * cols + x] == 0) d[(size_t)(rows - 1) * cols + x] = 0;
  }
}

}  // namespace

extern "C" int oracle_resize_u8(const uint8_t *src, int sw, int sh, uint8_t *dst, int dw, int dh) {
  if (!src || !dst || sw < 1 || sh < 1 || dw < 1 || dh < 1) return 1;
  resize_u8(src, sw, sh, dst, dw, dh);
  return 0;
}

extern "C" int oracle_hough_lines_p(const uint8_t *img, int width, int height, int threshold, int line_length,
                                    int line_gap, int32_t *lines_out, int capacity, int *count) {
  std::vector<Seg> lines;
  hough_lines_p(img, width, height, threshold, line_length, line_gap, lines);
  for (int k = 0; k < (int)lines.size() && k < capacity; ++k) {
    lines_out[4 * k] = lines[k].x0; lines_out[4 * k + 1] = lines[k].y0;
    lines_out[4 * k + 2] = lines[k].x1; lines_out[4 * k + 3] = lines[k].y1;
  }
  *count = (int)lines.size();
  return (int)lines.size() > capacity ? 2 : 0;
}

// EdgeSegment(scale, gray, 1, false, high_res_img) (DPE.cpp:136-291): the label map at the level
// size round(cols / 2^scale) x round(rows / 2^scale), -1 on small regions, 0 on edges.
extern "C" int oracle_edge_labels(const uint8_t *gray, int cols, int rows, int scale, int high_res_img,
                                  int32_t *labels_out, int out_cols, int out_rows) {
  const int robthr = high_res_img ? 4 : 6;
  const int weak_tex_num = (int)(1.0 * rows * cols / (1024 << scale << scale));
  std::vector<uint8_t> half;
  const uint8_t *s1 = gray;
  int c1 = cols, r1 = rows;
  if (high_res_img) {
    c1 = cols / 2; r1 = rows / 2;
    half.resize((size_t)c1 * r1);
    resize_u8(gray, cols, rows, half.data(), c1, r1);
    s1 = half.data();
  }
  const int c2 = c1 / 2, r2 = r1 / 2;
  std::vector<uint8_t> down((size_t)c2 * r2), dst((size_t)c2 * r2);
  resize_u8(s1, c1, r1, down.data(), c2, r2);
  const int m = c2 < r2 ? c2 : r2;
  const int houthr = (int)(m / 30.0), min_len = houthr, max_gap = houthr;
  roberts(down.data(), c2, r2, dst.data());
  for (auto &v : dst) v = v > robthr ? 255 : 0;
  std::vector<int32_t> lab0((size_t)c2 * r2), cnt0((size_t)c2 * r2 + 1);
  int n0 = 0;
  oracle_connect(dst.data(), c2, r2, lab0.data(), cnt0.data(), (int)cnt0.size(), &n0);
  std::vector<uint8_t> weak_img((size_t)c2 * r2);
  for (int k = 1; k < n0; ++k) {
    if (cnt0[k] < weak_tex_num) continue;
    for (int y = 0; y < r2; ++y)
      for (int x = 0; x < c2; ++x) {
        const size_t p = (size_t)y * c2 + x;
        weak_img[p] = 0;
        if (lab0[p] == k) continue;
        const bool border = (x > 0 && lab0[p - 1] == k) || (x < c2 - 1 && lab0[p + 1] == k) ||
                            (y > 0 && lab0[p - c2] == k) || (y < r2 - 1 && lab0[p + c2] == k);
        if (border) weak_img[p] = 255;
      }
    std::vector<Seg> lines;
    hough_lines_p(weak_img.data(), c2, r2, houthr, min_len, max_gap, lines);
    for (const Seg &l : lines) draw_line(dst.data(), c2, l.x0, l.y0, l.x1, l.y1);
  }
  const float factor = 1.0f / (float)(1 << scale);
  const int new_cols = (int)std::round(cols * factor), new_rows = (int)std::round(rows * factor);
  if (new_cols != out_cols || new_rows != out_rows) return 1;
  std::vector<uint8_t> up((size_t)new_cols * new_rows);
  if (new_cols == c2 && new_rows == r2) up = dst;
  else resize_u8(dst.data(), c2, r2, up.data(), new_cols, new_rows);
  for (auto &v : up) v = v > robthr ? 255 : 0;
  border_rule(up.data(), new_cols, new_rows);
  std::vector<int32_t> cnt((size_t)new_cols * new_rows + 1);
  int n = 0;
  oracle_connect(up.data(), new_cols, new_rows, labels_out, cnt.data(), (int)cnt.size(), &n);
  for (size_t p = 0; p < (size_t)new_cols * new_rows; ++p) {
    const int l = labels_out[p];
    if (l != 0 && cnt[l] <= weak_tex_num) labels_out[p] = -1;
  }
  return 0;
}
