// fzb_hfbook.cpp -- host construction of the canonical Huffman codebook used
// by the PHF coder (modules/coders/huffman/phf/hf_bk.cc:84-140,
// hf_bk_impl1.cc:73-163, hf_bk_internal.cc:59-101, hf_canon.cc:86-131).
//
// The reference builds this table on the host from the device histogram;
// so does this library (tens of microseconds for a thousand symbols: the
// heap's dependent loads set the pace).  The steps that fix the output bits:
//   * a 1-indexed binary min-heap: insertion stops at a parent whose
//     frequency is <= the new node's; removal moves the last node to the
//     root and sinks it, taking the right child only when strictly smaller
//     and swapping only when strictly larger;
//   * symbols enter the heap in increasing symbol order; each merge pops two
//     nodes and the FIRST popped becomes the RIGHT child (the reference's
//     host compiler evaluates the two pops of new_node(..., pop(), pop())
//     right to left);
//   * codes come from an iterative in-order walk (left = 0, right = 1) in a
//     64-bit book (58-bit code field, depth limit 58);
//   * lengths above 27 are replaced by the cutoff length 28 with code 0;
//   * canonical codes: first[l] = int((first[l+1] + numl[l+1]) / 2.0 + 0.5).
#include <cstdint>
#include <cstring>
#include <vector>

namespace fzb {

namespace {

struct Node {
    int left = -1, right = -1;
    uint64_t freq = 0;
    uint32_t sym = 0;
};

// The heap keeps each node's frequency beside its id, so a comparison reads
// one slot instead of following the id into the node array; the order of
// comparisons, and so every tie, is unchanged.
class MinHeap {
public:
    MinHeap() { slots_.push_back({0, -1}); }
    void reserve(size_t n) { slots_.reserve(n + 1); }
    size_t size() const { return slots_.size() - 1; }
    void push(int id, uint64_t freq) {
        slots_.push_back({freq, id});
        size_t i = slots_.size() - 1;
        while (i > 1) {
            const size_t parent = i >> 1;
            if (slots_[parent].freq <= freq) break;
            slots_[i] = slots_[parent];
            i = parent;
        }
        slots_[i] = {freq, id};
    }
    int pop() {
        const int top = slots_[1].id;
        const Slot moved = slots_.back();
        slots_.pop_back();
        const size_t end = slots_.size();
        if (end <= 1) return top;
        size_t i = 1;
        Slot* h = slots_.data();
        while (2 * i < end) {
            size_t c = 2 * i;
            // the right child only when strictly smaller (a select, not a branch)
            const uint64_t fl = h[c].freq;
            const uint64_t fr = c + 1 < end ? h[c + 1].freq : fl;
            c += fr < fl ? 1 : 0;
            if (!(moved.freq > h[c].freq)) break;
            h[i] = h[c];
            i = c;
        }
        h[i] = moved;
        return top;
    }

private:
    struct Slot {
        uint64_t freq;
        int id;
    };
    std::vector<Slot> slots_;
};

}  // namespace

// bk4: bklen words (bits 31..27 = length, low 27 = code; 0xffffffff =
// unused).  revbook: first[32] int | entry[32] int | keys u16[bklen].
// Returns 0, or -1 when the tree is deeper than the 58-level walk allows.
int build_huffman_book(const uint32_t* freq, uint32_t bklen, uint32_t* bk4, uint8_t* revbook) {
    std::vector<Node> nodes;
    nodes.reserve(2 * bklen + 2);
    for (uint32_t s = 0; s < bklen; s++)
        if (freq[s]) {
            Node nd;
            nd.freq = freq[s];
            nd.sym = s;
            nodes.push_back(nd);
        }
    MinHeap heap;
    heap.reserve(nodes.size());
    for (int i = 0; i < (int)nodes.size(); i++) heap.push(i, nodes[i].freq);
    while (heap.size() > 1) {
        const int right = heap.pop();
        const int left = heap.pop();
        Node nd;
        nd.left = left;
        nd.right = right;
        nd.freq = nodes[left].freq + nodes[right].freq;
        nodes.push_back(nd);
        heap.push((int)nodes.size() - 1, nd.freq);
    }

    std::vector<uint64_t> bk8(bklen, ~0ull);
    if (heap.size() == 1) {
        struct Frame { int node; uint64_t code, len; };
        std::vector<Frame> stack;
        int p = heap.pop();
        uint64_t code = 0, len = 0;
        while (true) {
            if (nodes[p].left >= 0 || nodes[p].right >= 0) {
                if (stack.size() + 1 > 58) return -1;
                stack.push_back({p, code, len});
                p = nodes[p].left;
                code <<= 1;
                if (++len > 58) return -1;
            } else {
                bk8[nodes[p].sym] = (code & ((1ull << 58) - 1)) | ((len & 63ull) << 58);
                if (stack.empty()) break;
                const Frame f = stack.back();
                stack.pop_back();
                p = nodes[f.node].right;
                code = (f.code << 1) | 1u;
                len = f.len + 1;
                if (len > 58) return -1;
            }
        }
    }

    // 64-bit -> 32-bit words: lengths above 27 become the cutoff 28, code 0
    for (uint32_t s = 0; s < bklen; s++) {
        if (bk8[s] == ~0ull) {
            bk4[s] = 0xffffffffu;
            continue;
        }
        uint32_t len = (uint32_t)(bk8[s] >> 58), code = (uint32_t)(bk8[s] & 0x7ffffffu);
        if (len > 27) {
            len = 28;
            code = 0;
        }
        bk4[s] = (len << 27) | code;
    }

    // canonical form
    int numl[32] = {0}, entry[32] = {0}, first[32] = {0}, next[32];
    int max_l = 0;
    for (uint32_t s = 0; s < bklen; s++)
        if (bk4[s] != 0xffffffffu) {
            const int l = (int)(bk4[s] >> 27);
            numl[l]++;
            if (l > max_l) max_l = l;
        }
    for (int i = 1; i < 32; i++) entry[i] = entry[i - 1] + numl[i - 1];
    for (int i = 0; i < 32; i++) next[i] = entry[i];
    first[max_l] = 0;
    for (int l = max_l - 1; l >= 1; l--) first[l] = (int)((first[l + 1] + numl[l + 1]) / 2.0 + 0.5);
    first[0] = 0xff;
    std::vector<uint16_t> keys(bklen, 0);
    std::vector<uint32_t> canon(bklen, 0xffffffffu);
    for (uint32_t s = 0; s < bklen; s++) {
        const uint32_t w = bk4[s];
        if (w == 0xffffffffu) continue;
        const uint32_t l = w >> 27;
        const int slot = next[l]++;
        canon[slot] = ((uint32_t)(first[l] + slot - entry[l]) & 0x7ffffffu) | (l << 27);
        keys[slot] = (uint16_t)s;
    }
    for (uint32_t s = 0; s < bklen; s++) bk4[s] = 0xffffffffu;
    for (uint32_t i = 0; i < bklen; i++)
        if (canon[i] != 0xffffffffu) bk4[keys[i]] = canon[i];
    std::memcpy(revbook, first, sizeof(first));
    std::memcpy(revbook + sizeof(first), entry, sizeof(entry));
    std::memcpy(revbook + 2 * sizeof(first), keys.data(), 2 * (size_t)bklen);
    return 0;
}

}  // namespace fzb
