};  // struct RefDetail
}  // namespace libraw_enhanced

/* ref_detail_suffix.h -- TEST INFRASTRUCTURE.  C ABI over the streamed
 * apply_detail_preserving_tonemap: rgb is (H, W, 3) float, updated in place.
 * std::cout is muted for the call unless LRE_REF_VERBOSE is set. */
extern "C" int ref_detail_tonemap(float* rgb, size_t w, size_t h) {
  std::streambuf* saved = nullptr;
  if (!std::getenv("LRE_REF_VERBOSE")) saved = std::cout.rdbuf(nullptr);
  libraw_enhanced::ImageBufferFloat buf;
  buf.image = reinterpret_cast<float (*)[3]>(rgb);
  buf.width = w;
  buf.height = h;
  buf.channels = 3;
  libraw_enhanced::RefDetail r;
  r.apply_detail_preserving_tonemap(buf);
  if (saved) {
    std::cout.rdbuf(saved);
    std::cout.clear();
  }
  return 1;
}
