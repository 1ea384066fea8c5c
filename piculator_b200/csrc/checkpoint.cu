// Checkpoint / resume of a pi computation.
//
// The reference keeps everything in RAM and restarts from nothing after a
// failure ("Memory Mode: RAM", PI.h:165-166).  Here a computation can write
// its state at the end of each phase of Pi() (PI.h:179-194) and a later call
// for the same digit count can resume from the newest state on disk:
//   phase 1: binary splitting done, P = 13591409 Q + P, Q = 4270934400 Q
//            (PI.h:179-181): the two BigFloats P, Q;
//   phase 2: division done, P = Q / P (PI.h:189): P;
//   phase 3: inverse square root done, Q = invsqrt(10005) (PI.h:194): P, Q.
// The final product and the text follow from phase 3 in a fraction of the
// run.  Binary splitting is about 90 % of the device time, so phase 1 saves
// most of a run; the state is two numbers of p + 2 words.
//
// File <dir>/pi_<digits>.ckpt, little-endian:
//   char magic[8] = "PICKPT01"
//   uint64 digits, p_words, terms
//   uint32 phase, uint32 count
//   count x { int32 sign, int32 pad, int64 exp, uint64 L, uint64 hash }
//   the words of the count numbers, in order
// hash = ckpt_hash over the number's words (see below); a file whose header
// or hashes do not match, or whose length fields do not add up to the file's
// size, is rejected (PIC_ERR_IO), never used.  A new file is written beside
// the old one, flushed to disk and renamed over it, so a crash while writing
// leaves the previous checkpoint intact.
#include <errno.h>
#include <stdio.h>
#include <string.h>
#include <unistd.h>

#include <string>
#include <vector>

#include "bigfloat.hpp"
#include "checkpoint.cuh"
#include "common.cuh"

namespace pic {

static std::string g_dir;
static int g_flags = 0;
static int g_stop_after = 0;

void checkpoint_configure(const char* dir, int flags)
{
    g_dir = dir ? dir : "";
    g_flags = dir ? flags : 0;
}

void checkpoint_debug_stop_after(int phase) { g_stop_after = phase; }

uint64_t ckpt_hash(const uint32_t* w, size_t n)
{
    // 64-bit multiply-xorshift over 32-bit words, seeded with the length
    uint64_t h = 0x243F6A8885A308D3ull ^ (uint64_t)n;
    for (size_t i = 0; i < n; i++) {
        h = (h ^ w[i]) * 0x9E3779B97F4A7C15ull;
        h ^= h >> 29;
    }
    return h;
}

namespace {
struct Header {
    char magic[8];
    uint64_t digits, p_words, terms;
    uint32_t phase, count;
};
struct Entry {
    int32_t sign, pad;
    int64_t exp;
    uint64_t L, hash;
};
constexpr char kMagic[8] = {'P', 'I', 'C', 'K', 'P', 'T', '0', '1'};
constexpr uint32_t kMaxCount = 4;

std::string file_for(uint64_t digits) { return g_dir + "/pi_" + std::to_string(digits) + ".ckpt"; }

struct File {
    FILE* f = nullptr;
    explicit File(FILE* x) : f(x) {}
    ~File()
    {
        if (f) fclose(f);
    }
};

[[noreturn]] void io_error(const std::string& what, const std::string& path)
{
    throw Error(PIC_ERR_IO, "checkpoint " + path + ": " + what);
}
}  // namespace

int checkpoint_inspect_file(const char* path, uint64_t* digits, uint64_t* p_words, uint32_t* phase, bool verify,
                            std::vector<CkptNumber>* numbers)
{
    File f(fopen(path, "rb"));
    if (!f.f) return -1;
    Header h;
    if (fread(&h, sizeof h, 1, f.f) != 1 || memcmp(h.magic, kMagic, 8) != 0) io_error("not a checkpoint file", path);
    if (h.phase < 1 || h.phase > 3 || h.count < 1 || h.count > kMaxCount) io_error("bad phase or count", path);
    std::vector<Entry> ent(h.count);
    if (fread(ent.data(), sizeof(Entry), h.count, f.f) != h.count) io_error("truncated header", path);
    if (digits) *digits = h.digits;
    if (p_words) *p_words = h.p_words;
    if (phase) *phase = h.phase;
    if (!verify) return 0;
    // the words must fill the rest of the file exactly: checked before any
    // buffer is sized from a length field, so a damaged length cannot ask
    // for an enormous allocation
    uint64_t want = 0;
    for (uint32_t i = 0; i < h.count; i++) {
        if (ent[i].L > ((uint64_t)1 << 36)) io_error("bad length", path);
        want += 4 * ent[i].L;
    }
    const long pos = ftell(f.f);
    if (pos < 0 || fseek(f.f, 0, SEEK_END) != 0) io_error("cannot seek", path);
    const long end = ftell(f.f);
    if (end < pos || fseek(f.f, pos, SEEK_SET) != 0) io_error("cannot seek", path);
    if ((uint64_t)(end - pos) < want) io_error("truncated words", path);
    if ((uint64_t)(end - pos) > want) io_error("trailing bytes", path);
    for (uint32_t i = 0; i < h.count; i++) {
        std::vector<uint32_t> w(ent[i].L);
        if (ent[i].L && fread(w.data(), 4, ent[i].L, f.f) != ent[i].L) io_error("truncated words", path);
        if (ckpt_hash(w.data(), w.size()) != ent[i].hash) io_error("words do not match their hash", path);
        if (numbers) numbers->push_back(CkptNumber{ent[i].sign != 0, ent[i].exp, std::move(w)});
    }
    if (fgetc(f.f) != EOF) io_error("trailing bytes", path);
    return 0;
}

int checkpoint_resume(uint64_t digits, uint64_t p_words, BigFloat* P, BigFloat* Q)
{
    if (g_dir.empty() || !(g_flags & PIC_CKPT_RESUME)) return 0;
    const std::string path = file_for(digits);
    std::vector<CkptNumber> nums;
    uint64_t d = 0, pw = 0;
    uint32_t phase = 0;
    if (checkpoint_inspect_file(path.c_str(), &d, &pw, &phase, true, &nums) != 0) return 0;  // none yet
    if (d != digits || pw != p_words) io_error("written for another computation", path);
    const size_t want = phase == 2 ? 1 : 2;
    if (nums.size() != want) io_error("wrong number count for its phase", path);
    auto load = [](const CkptNumber& n) { return BigFloat::from_host(n.sign, n.exp, n.words.data(), n.words.size()); };
    *P = load(nums[0]);
    if (want == 2) *Q = load(nums[1]);
    return (int)phase;
}

void checkpoint_save(int phase, uint64_t digits, uint64_t p_words, uint64_t terms, const BigFloat* P,
                     const BigFloat* Q)
{
    if (g_dir.empty() || !(g_flags & PIC_CKPT_WRITE)) return;
    const std::string path = file_for(digits), tmp = path + ".tmp";
    std::vector<const BigFloat*> nums{P};
    if (Q) nums.push_back(Q);
    std::vector<std::vector<uint32_t>> words;
    std::vector<Entry> ent;
    for (const BigFloat* x : nums) {
        words.push_back(x->words());
        Entry e{};
        e.sign = x->get_sign() ? 1 : 0;
        e.exp = x->get_exponent();
        e.L = x->get_precision();
        e.hash = ckpt_hash(words.back().data(), words.back().size());
        ent.push_back(e);
    }
    Header h{};
    memcpy(h.magic, kMagic, 8);
    h.digits = digits;
    h.p_words = p_words;
    h.terms = terms;
    h.phase = (uint32_t)phase;
    h.count = (uint32_t)nums.size();
    {
        File f(fopen(tmp.c_str(), "wb"));
        if (!f.f) io_error(std::string("cannot create (") + strerror(errno) + ")", tmp);  // PI.h:42
        bool ok = fwrite(&h, sizeof h, 1, f.f) == 1 && fwrite(ent.data(), sizeof(Entry), ent.size(), f.f) == ent.size();
        for (const auto& w : words) ok = ok && (w.empty() || fwrite(w.data(), 4, w.size(), f.f) == w.size());
        // on disk before the rename, so the name never points at a file
        // whose data a system crash could still lose
        ok = ok && fflush(f.f) == 0 && fsync(fileno(f.f)) == 0;
        if (!ok) io_error("write failed", tmp);
    }
    if (rename(tmp.c_str(), path.c_str()) != 0) io_error(std::string("rename failed (") + strerror(errno) + ")", path);
    if (g_stop_after == phase)
        throw Error(PIC_ERR_STOPPED, "stopped after writing the checkpoint of phase " + std::to_string(phase));
}

}  // namespace pic
