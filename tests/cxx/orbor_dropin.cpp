// Drop-in check of the C++ API (include/orb.h, include/orbd.h): the call
// sequence of the reference demo (main.cpp:177-243) plus the lower-level
// orbd.h pipeline on caller-owned buffers (orb.cpp:57-101, 145-201).
//
// usage: orbor_dropin <w> <h> <imgA.raw> <imgB.raw> <out.bin> <max_pts>
// images: h rows of align_up(w,128) bytes.  out.bin: for A and B, num_pts then
// num_pts OrbPoint and num_pts*32 descriptor bytes (Orbor path), then the
// match/distance of A, then the same keypoints/descriptors from the lower API.
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "orb.h"
#include "orbd.h"

static std::vector<unsigned char> read_file(const char* path, size_t n) {
  std::vector<unsigned char> v(n);
  FILE* f = std::fopen(path, "rb");
  if (!f || std::fread(v.data(), 1, n, f) != n) {
    std::fprintf(stderr, "cannot read %s\n", path);
    std::exit(2);
  }
  std::fclose(f);
  return v;
}

static void write_result(FILE* f, orb::OrbData& d, unsigned char* d_desc) {
  std::fwrite(&d.num_pts, sizeof(int), 1, f);
  std::vector<orb::OrbPoint> pts(d.num_pts > 0 ? d.num_pts : 1);
  std::vector<unsigned char> desc((size_t)(d.num_pts > 0 ? d.num_pts : 1) * 32);
  if (d.num_pts > 0) {
    CHECK(cudaMemcpy(pts.data(), d.d_data, sizeof(orb::OrbPoint) * d.num_pts, cudaMemcpyDeviceToHost));
    CHECK(cudaMemcpy(desc.data(), d_desc, 32 * (size_t)d.num_pts, cudaMemcpyDeviceToHost));
    std::fwrite(pts.data(), sizeof(orb::OrbPoint), d.num_pts, f);
    std::fwrite(desc.data(), 1, 32 * (size_t)d.num_pts, f);
  }
}

int main(int argc, char** argv) {
  if (argc < 7) return 2;
  const int w = std::atoi(argv[1]), h = std::atoi(argv[2]);
  const int max_pts = std::atoi(argv[6]);
  const int pitch = iAlignUp(w, 128);
  std::vector<unsigned char> ha = read_file(argv[3], (size_t)h * pitch);
  std::vector<unsigned char> hb = read_file(argv[4], (size_t)h * pitch);
  if (!initDevice(0)) return 3;
  unsigned char *img1 = NULL, *img2 = NULL;
  CHECK(cudaMalloc((void**)&img1, (size_t)h * pitch));
  CHECK(cudaMalloc((void**)&img2, (size_t)h * pitch));
  CHECK(cudaMemcpy(img1, ha.data(), ha.size(), cudaMemcpyHostToDevice));
  CHECK(cudaMemcpy(img2, hb.data(), hb.size(), cudaMemcpyHostToDevice));
  int3 whp = make_int3(w, h, pitch);

  // --- the demo's sequence through orb::Orbor ---
  orb::Orbor det;
  det.init(8, 31, 2, orb::HARRIS_SCORE, 31, 20, -1, max_pts);
  orb::OrbData d1, d2;
  det.initOrbData(d1, max_pts, true, true);
  det.initOrbData(d2, max_pts, true, true);
  unsigned char *desc1 = NULL, *desc2 = NULL;
  for (int rep = 0; rep < 2; rep++) {
    det.detectAndCompute(img1, d1, whp, (void**)&desc1, true);
    det.detectAndCompute(img2, d2, whp, (void**)&desc2, true);
    det.match(d1, d2, desc1, desc2);
  }
  FILE* f = std::fopen(argv[5], "wb");
  write_result(f, d1, desc1);
  write_result(f, d2, desc2);
  for (int i = 0; i < d1.num_pts; i++) {
    std::fwrite(&d1.h_data[i].match, sizeof(int), 1, f);
    std::fwrite(&d1.h_data[i].distance, sizeof(int), 1, f);
  }

  // --- the lower orbd.h API on caller-owned pyramid and score buffers ---
  orb::setMaxNumPoints(max_pts);
  orb::setFastThresholdLUT(20);
  orb::setUmax(31);
  orb::setPattern(31, 2);
  orb::setGaussianKernel();
  orb::setScaleSqSq();
  unsigned int* counter = NULL;
  orb::getPointCounter((void**)&counter);
  // layout as Orbor::updateParam computes it (orb.cpp:148-174)
  int n = 8, m = (w < h ? w : h) / 80, lv = 0;
  while ((1 << lv) <= m) lv++;
  if (lv < n) n = lv;
  std::vector<int> oszp(5 * n + 1);
  int *osizes = oszp.data(), *widths = osizes + n, *heights = widths + n, *pitchs = heights + n,
      *offsets = pitchs + n;
  widths[0] = w;
  heights[0] = h;
  pitchs[0] = pitch;
  osizes[0] = h * pitch;
  offsets[0] = 0;
  offsets[1] = osizes[0];
  for (int j = 1; j < n; j++) {
    widths[j] = widths[j - 1] >> 1;
    heights[j] = heights[j - 1] >> 1;
    pitchs[j] = iAlignUp(widths[j], 128);
    osizes[j] = heights[j] * pitchs[j];
    offsets[j + 1] = offsets[j] + osizes[j];
  }
  unsigned char* omem = NULL;
  float* vmem = NULL;
  CHECK(cudaMalloc((void**)&omem, offsets[n]));
  CHECK(cudaMalloc((void**)&vmem, (size_t)osizes[0] * 8));
  orb::makeOffsets(pitchs, n);
  orb::OrbData l1;
  det.initOrbData(l1, max_pts, true, true);
  unsigned char* ldesc = NULL;
  CHECK(cudaMalloc((void**)&ldesc, (size_t)max_pts * 32));
  for (int img = 0; img < 2; img++) {
    CHECK(cudaMemset(counter, 0, sizeof(unsigned int)));
    orb::hFastDectectWithNMS(img == 0 ? img1 : img2, omem, vmem, l1, oszp.data(), n, 20, 31, true);
    unsigned int cnt = 0;
    CHECK(cudaMemcpy(&cnt, counter, sizeof(unsigned int), cudaMemcpyDeviceToHost));
    l1.num_pts = (int)cnt < max_pts ? (int)cnt : max_pts;
    orb::hComputeAngle(omem, l1, oszp.data(), n, 31);
    orb::hGassianBlur(omem, oszp.data(), n);
    orb::hDescribe(omem, l1, ldesc, 2, n);
    write_result(f, l1, ldesc);
  }
  std::fclose(f);
  det.freeOrbData(d1);
  det.freeOrbData(d2);
  det.freeOrbData(l1);
  std::printf("ok %d %d\n", d1.num_pts, d2.num_pts);
  return 0;
}
