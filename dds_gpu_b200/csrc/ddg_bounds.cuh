// Cheap trick bounds at the start of a trick and for the second hand: DDS QuickTricks,
// QuickTricksSecondHand and LaterTricks (MIN/MAX), as the reference runs them
// (src/dd_bounds.h:11-584, itself a port of DDS quick_tricks.cpp / later_tricks.cpp by
// Bo Haglund and Soren Hein, Apache-2.0). The decisions and their order are the DDS
// algorithm and are kept step for step, because every bound that fires changes which
// nodes the search visits; the data layout is new: the per-suit top-card table lives in
// a few packed registers instead of small arrays indexed at run time.
#pragma once
#include "ddg_bits.cuh"

namespace ddg {

// Top three cards of every suit with their holders, plus all suit lengths.
struct Top {
  u64 lens;                 // length_key() layout
  u32 win_h, sec_h, thr_h;  // byte s: holder of the 1st/2nd/3rd card of suit s, 0xFF = none
  u32 win_c, sec_c, thr_c;  // byte s: that card (0 when none)
};

DDG_HD int sbyte(u32 x, int s) { return (int)(int8_t)(uint8_t)(x >> (8 * s)); }
DDG_HD int ubyte(u32 x, int s) { return (int)((x >> (8 * s)) & 0xFF); }
DDG_HD int tlen(const Top& t, int h, int s) { return len_of(t.lens, h, s); }
DDG_HD int winh(const Top& t, int s) { return sbyte(t.win_h, s); }
DDG_HD int sech(const Top& t, int s) { return sbyte(t.sec_h, s); }
DDG_HD int thrh(const Top& t, int s) { return sbyte(t.thr_h, s); }
DDG_HD int winc(const Top& t, int s) { return ubyte(t.win_c, s); }
DDG_HD int secc(const Top& t, int s) { return ubyte(t.sec_c, s); }
DDG_HD int thrc(const Top& t, int s) { return ubyte(t.thr_c, s); }

// src/dd_bounds.h:18-32: lengths from `lens`, top three cards of each suit (missing card:
// holder -1, card 0).
DDG_CALL Top make_top(Hands hs, u64 lens) {
  const u64* h = hs.h;
  Top t;
  t.lens = lens;
  t.win_h = t.sec_h = t.thr_h = 0;
  t.win_c = t.sec_c = t.thr_c = 0;
  u64 all = all_cards(h);
#pragma unroll
  for (int s = 0; s < 4; s++) {
    u64 a = all & suit_cards(s);
    u32 who[3], crd[3];
#pragma unroll
    for (int k = 0; k < 3; k++) {
      int c = a ? top_bit(a) : 0;
      who[k] = a ? (u32)holder_of(h, c) : 0xFFu;
      crd[k] = (u32)c;
      a &= ~card_bit(c);
    }
    t.win_h |= who[0] << (8 * s);
    t.sec_h |= who[1] << (8 * s);
    t.thr_h |= who[2] << (8 * s);
    t.win_c |= crd[0] << (8 * s);
    t.sec_c |= crd[1] << (8 * s);
    t.thr_c |= crd[2] << (8 * s);
  }
  return t;
}

struct QtOut {  // QuickTricks: count, whether it decided the node, the cards that did
  int q, decided;
  u64 wr;
};
struct BoundOut {  // a bound's answer and the cards that decided it
  int v;
  u64 wr;
};

// Suit order of QuickTricks: trumps first, then the side suits in order.
DDG_HD int qt_next_suit(int suit, int trump) {
  if (trump >= 0 && suit == trump) return trump == 0 ? 1 : 0;
  suit++;
  if (trump >= 0 && suit == trump) suit++;
  return suit;
}

// Outcome of one suit's quick tricks: keep going in the suit, stop (cutoff reached), or
// go to the next suit.
enum { QT_STAY = 0, QT_STOP = 1, QT_NEXT = 2 };

struct QtSuit {  // the counts of one suit as QuickTricks sees them
  int own, part, lho, rho;
};

// Leader holds the top card of a side suit, trumps out (DDS QtricksLeadHandTrump).
DDG_HD int qt_lead_side(const Top& t, int hand, int cutoff, QtSuit c, int lhoT, int rhoT,
                        int suit, int qt, u64& wr, int& res) {
  int P = partner_of(hand);
  res = QT_STOP;
  if ((c.lho != 0 || lhoT == 0) && (c.rho != 0 || rhoT == 0)) {
    wr |= card_bit(winc(t, suit));
    if (++qt >= cutoff) return qt;
    if (c.lho <= 1 && c.rho <= 1 && c.part <= 1 && lhoT == 0 && rhoT == 0) {
      qt += c.own - 1;
      if (qt >= cutoff) return qt;
      res = QT_NEXT;
      return qt;
    }
  }
  int s2 = sech(t, suit);
  if (s2 == hand) {
    if (lhoT == 0 && rhoT == 0) {
      wr |= card_bit(secc(t, suit));
      if (++qt >= cutoff) return qt;
      if (c.lho <= 2 && c.rho <= 2 && c.part <= 2) {
        qt += c.own - 2;
        if (qt >= cutoff) return qt;
        res = QT_NEXT;
        return qt;
      }
    }
  } else if (s2 == P && c.own > 1 && c.part > 1) {
    if (lhoT == 0 && rhoT == 0) {
      wr |= card_bit(secc(t, suit));
      if (++qt >= cutoff) return qt;
      if (c.lho <= 2 && c.rho <= 2 && (c.part <= 2 || c.own <= 2)) {
        qt += (c.own > c.part ? c.own : c.part) - 2;
        if (qt >= cutoff) return qt;
        res = QT_NEXT;
        return qt;
      }
    }
  }
  res = QT_STAY;
  return qt;
}

// Leader holds the top card, no trump issue (NT, or the trump suit itself): DDS
// QtricksLeadHandNT. Cashing trumps draws the opponents' trumps (lhoT/rhoT).
DDG_HD int qt_lead_plain(const Top& t, int hand, int cutoff, QtSuit c, int& lhoT, int& rhoT,
                         bool comm, int comm_suit, int suit, int qt, int trump, u64& wr,
                         int& res) {
  int P = partner_of(hand);
  bool draws = trump == suit && (!comm || suit != comm_suit);
  res = QT_STOP;
  wr |= card_bit(winc(t, suit));
  if (++qt >= cutoff) return qt;
  if (draws) {
    lhoT = lhoT > 0 ? lhoT - 1 : 0;
    rhoT = rhoT > 0 ? rhoT - 1 : 0;
  }
  if (c.lho <= 1 && c.rho <= 1 && c.part <= 1) {
    qt += c.own - 1;
    if (qt >= cutoff) return qt;
    res = QT_NEXT;
    return qt;
  }
  int s2 = sech(t, suit);
  if (s2 == hand) {
    wr |= card_bit(secc(t, suit));
    if (++qt >= cutoff) return qt;
    if (draws) {
      lhoT = lhoT > 0 ? lhoT - 1 : 0;
      rhoT = rhoT > 0 ? rhoT - 1 : 0;
    }
    if (c.lho <= 2 && c.rho <= 2 && c.part <= 2) {
      qt += c.own - 2;
      if (qt >= cutoff) return qt;
      res = QT_NEXT;
      return qt;
    }
  } else if (s2 == P && c.own > 1 && c.part > 1) {
    wr |= card_bit(secc(t, suit));
    if (++qt >= cutoff) return qt;
    if (draws) {
      lhoT = lhoT > 0 ? lhoT - 1 : 0;
      rhoT = rhoT > 0 ? rhoT - 1 : 0;
    }
    if (c.lho <= 2 && c.rho <= 2 && (c.part <= 2 || c.own <= 2)) {
      qt += (c.own > c.part ? c.own : c.part) - 2;
      if (qt >= cutoff) return qt;
      res = QT_NEXT;
      return qt;
    }
  }
  res = QT_STAY;
  return qt;
}

// Partner holds the top card of a side suit and the leader can reach partner
// (DDS QtricksLeadHandTrump for partner's suit).
DDG_HD int qt_partner_side(const Top& t, int hand, int cutoff, QtSuit c, int lhoT, int rhoT,
                           int suit, int qt, int comm_suit, int comm_card, u64& wr, int& res) {
  int P = partner_of(hand), L = lho_of(hand);
  u64 entry = card_bit(comm_card);
  res = QT_STOP;
  if ((c.lho != 0 || lhoT == 0) && (c.rho != 0 || rhoT == 0)) {
    wr |= card_bit(winc(t, suit)) | entry;
    if (++qt >= cutoff) return qt;
    if (c.lho <= 1 && c.rho <= 1 && c.own <= 1 && lhoT == 0 && rhoT == 0) {
      qt += c.part - 1;
      if (qt >= cutoff) return qt;
      res = QT_NEXT;
      return qt;
    }
  }
  int s2 = sech(t, suit);
  if (s2 == P) {
    if (lhoT == 0 && rhoT == 0) {
      wr |= card_bit(secc(t, suit)) | entry;
      if (++qt >= cutoff) return qt;
      if (c.lho <= 2 && c.rho <= 2 && c.own <= 2) {
        qt += c.part - 2;
        if (qt >= cutoff) return qt;
        res = QT_NEXT;
        return qt;
      }
    }
  } else if (s2 == hand && c.part > 1 && c.own > 1) {
    if (lhoT == 0 && rhoT == 0) {
      wr |= card_bit(secc(t, suit)) | entry;
      if (++qt >= cutoff) return qt;
      if (c.lho <= 2 && c.rho <= 2 && (c.own <= 2 || c.part <= 2)) {
        qt += (c.part > c.own ? c.part : c.own) - 2;
        if (qt >= cutoff) return qt;
        res = QT_NEXT;
        return qt;
      }
    }
  } else if (suit == comm_suit && s2 == L && (c.lho >= 2 || lhoT == 0) && (c.rho >= 2 || rhoT == 0)) {
    if (thrh(t, suit) == P) {
      wr |= card_bit(thrc(t, suit)) | entry;
      if (++qt >= cutoff) return qt;
      if (c.own <= 2 && c.lho <= 2 && c.rho <= 2 && lhoT == 0 && rhoT == 0) {
        qt += c.part - 2;
        if (qt >= cutoff) return qt;
      }
    }
  }
  res = QT_STAY;
  return qt;
}

// Partner holds the top card, no trump issue (DDS QtricksLeadHandNT for partner's suit).
DDG_HD int qt_partner_plain(const Top& t, int hand, int cutoff, QtSuit c, int suit, int qt,
                            int comm_suit, int comm_card, u64& wr, int& res) {
  int P = partner_of(hand), L = lho_of(hand);
  res = QT_STOP;
  wr |= card_bit(winc(t, suit)) | card_bit(comm_card);
  if (++qt >= cutoff) return qt;
  if (c.lho <= 1 && c.rho <= 1 && c.own <= 1) {
    qt += c.part - 1;
    if (qt >= cutoff) return qt;
    res = QT_NEXT;
    return qt;
  }
  int s2 = sech(t, suit);
  if (s2 == P) {
    wr |= card_bit(secc(t, suit));
    if (++qt >= cutoff) return qt;
    if (c.lho <= 2 && c.rho <= 2 && c.own <= 2) {
      qt += c.part - 2;
      if (qt >= cutoff) return qt;
      res = QT_NEXT;
      return qt;
    }
  } else if (s2 == hand && c.part > 1 && c.own > 1) {
    wr |= card_bit(secc(t, suit));
    if (++qt >= cutoff) return qt;
    if (c.lho <= 2 && c.rho <= 2 && (c.own <= 2 || c.part <= 2)) {
      qt += (c.part > c.own ? c.part : c.own) - 2;
      if (qt >= cutoff) return qt;
      res = QT_NEXT;
      return qt;
    }
  } else if (suit == comm_suit && s2 == L) {
    if (thrh(t, suit) == P) {
      wr |= card_bit(thrc(t, suit));
      if (++qt >= cutoff) return qt;
      if (c.own <= 2 && c.lho <= 2 && c.rho <= 2) {
        qt += c.part - 2;
        if (qt >= cutoff) return qt;
      }
    }
  }
  res = QT_STAY;
  return qt;
}

// A suit where neither opponent follows decides at once if the sure length of the
// partnership's suit already reaches the cutoff (the two "sum" tests of DDS QuickTricks;
// `lead_side` = the leader is the longer or equal hand).
DDG_HD int qt_blocked_sum(const Top& t, int hand, int trump, int suit, QtSuit c, int lhoT,
                          int rhoT, bool lead_side, int cutoff, bool& hit) {
  int P = partner_of(hand);
  hit = false;
  if (trump >= 0 && suit == trump) {
    int sum = c.own > c.part ? c.own : c.part;
    for (int s = 0; s < 4; s++) {
      bool shortness = lead_side ? (c.own >= c.part && tlen(t, hand, s) > 0 && tlen(t, P, s) == 0)
                                 : (c.own <= c.part && tlen(t, P, s) > 0 && tlen(t, hand, s) == 0);
      if (sum > 0 && s != trump && shortness) {
        sum++;
        break;
      }
    }
    hit = sum >= cutoff;
    return sum;
  }
  int sum = c.own < c.part ? c.own : c.part;
  if (trump < 0 || (suit != trump && lhoT == 0 && rhoT == 0)) hit = sum >= cutoff;
  return sum;
}

// DDS QuickTricks for the side on lead (src/dd_bounds.h:245-438). `cutoff` = tricks the
// leading side needs; `decided` = true when the answer is known: a count > 0 means the
// leading side makes it, 0 that it fails (the opponents need `cutoff_other`).
DDG_HD int quick_tricks_impl(const u64* hands, const Top& t, int trump, int hand, int cutoff,
                        int cutoff_other, u64& wr, bool& decided) {
  const int P = partner_of(hand), L = lho_of(hand), R = rho_of(hand);
  int comm_card = 0, comm_suit = -1, qtricks = 0;
  bool comm = false, ruffed = false;
  decided = true;

  // An entry to partner in a side suit: partner's top card of a suit the leader holds, or
  // partner's second card behind the leader's top card; with trumps, only where neither
  // opponent can ruff. The first suit that gives one is taken.
  for (int s = 0; s < 4 && !comm; s++) {
    if (trump >= 0 && s == trump) continue;
    bool safe = trump < 0 || ((tlen(t, L, s) != 0 || tlen(t, L, trump) == 0) &&
                              (tlen(t, R, s) != 0 || tlen(t, R, trump) == 0));
    if (winh(t, s) == P) {
      if (tlen(t, hand, s) != 0 && safe) {
        comm = true;
        comm_suit = s;
        comm_card = winc(t, s);
      }
    } else if (sech(t, s) == P && winh(t, s) == hand && tlen(t, hand, s) >= 2 &&
               tlen(t, P, s) >= 2 && safe) {
      comm = true;
      comm_suit = s;
      comm_card = secc(t, s);
    }
  }
  if (trump >= 0 && !comm && tlen(t, hand, trump) != 0 && winh(t, trump) == P) {
    comm = true;
    comm_suit = trump;
    comm_card = winc(t, trump);
  }

  int lhoT = 0, rhoT = 0, suit = 0;
  if (trump >= 0) {
    suit = trump;
    lhoT = tlen(t, L, trump);
    rhoT = tlen(t, R, trump);
  }
  do {
    QtSuit c;
    c.own = tlen(t, hand, suit);
    c.lho = tlen(t, L, suit);
    c.rho = tlen(t, R, suit);
    c.part = tlen(t, P, suit);
    bool opps = (c.lho | c.rho) != 0;
    if (!opps && c.part == 0) {
      // Only the leader holds the suit: long tricks, unless an opponent can ruff.
      if (c.own != 0 && (trump < 0 || trump == suit || (lhoT == 0 && rhoT == 0))) {
        qtricks += c.own;
        if (qtricks >= cutoff) return qtricks;
      }
      suit = qt_next_suit(suit, trump);
      continue;
    }
    if (!opps) {
      bool hit;
      int sum = qt_blocked_sum(t, hand, trump, suit, c, lhoT, rhoT, true, cutoff, hit);
      if (hit) return sum;
    }
    if (comm) {
      if (!opps && c.own == 0) {
        // Only partner holds the suit: cash it over the entry.
        if (trump < 0 || trump == suit || (lhoT == 0 && rhoT == 0)) {
          qtricks += c.part;
          wr |= card_bit(comm_card);
          if (qtricks >= cutoff) return qtricks;
        }
        suit = qt_next_suit(suit, trump);
        continue;
      }
      if (!opps) {
        bool hit;
        int sum = qt_blocked_sum(t, hand, trump, suit, c, lhoT, rhoT, false, cutoff, hit);
        if (hit) {
          if (trump >= 0 && suit == trump) wr |= card_bit(comm_card);
          return sum;
        }
      }
    }
    int w = winh(t, suit);
    if (w < 0) {
      suit = qt_next_suit(suit, trump);
      continue;
    }
    int res = QT_STAY;
    bool side = trump >= 0 && trump != suit;
    if (w == hand) {
      qtricks = side ? qt_lead_side(t, hand, cutoff, c, lhoT, rhoT, suit, qtricks, wr, res)
                     : qt_lead_plain(t, hand, cutoff, c, lhoT, rhoT, comm, comm_suit, suit,
                                     qtricks, trump, wr, res);
    } else if (w == P && comm) {
      qtricks = side ? qt_partner_side(t, hand, cutoff, c, lhoT, rhoT, suit, qtricks, comm_suit,
                                       comm_card, wr, res)
                     : qt_partner_plain(t, hand, cutoff, c, suit, qtricks, comm_suit, comm_card,
                                        wr, res);
    }
    if (res == QT_STOP) return qtricks;
    if (res == QT_NEXT) {
      suit = qt_next_suit(suit, trump);
      continue;
    }

    // A ruff by partner: the leader leads the suit and partner, void, trumps it.
    if (side && c.own > 0 && !ruffed &&
        (qtricks == 0 || (w != hand && w != P && winh(t, trump) != hand && winh(t, trump) != P))) {
      if (c.part == 0 && tlen(t, P, trump) > 0) {
        u64 T = suit_cards(trump);
        u64 pt = hand_at(hands, P) & T;
        if ((c.rho > 0 || tlen(t, R, trump) == 0) && (c.lho > 0 || tlen(t, L, trump) == 0)) {
          ruffed = true;  // nobody can overruff
          if (1 >= cutoff) return 1;
          suit = qt_next_suit(suit, trump);
          continue;
        }
        u64 over = 0;  // trumps of the opponents that are void in the suit
        if (c.lho == 0) over |= hand_at(hands, L) & T;
        if (c.rho == 0) over |= hand_at(hands, R) & T;
        if (over < pt) {
          ruffed = true;
          wr |= card_bit(top_bit(pt));
          if (1 >= cutoff) return 1;
        }
        suit = qt_next_suit(suit, trump);
        continue;
      }
    }
    if (qtricks >= cutoff) return qtricks;
    suit = qt_next_suit(suit, trump);
  } while (suit <= 3);

  if (qtricks == 0 && (trump < 0 || winh(t, trump) < 0)) {
    // No quick trick: the opponents win the first trick with a top card.
    for (int s = 0; s < 4; s++) {
      if (winh(t, s) < 0) continue;
      if (tlen(t, hand, s) > 0) wr = (wr & ~suit_cards(s)) | card_bit(winc(t, s));
    }
    if (1 >= cutoff_other) return 0;
  }
  decided = false;
  return qtricks;
}

// DDS QuickTricksSecondHand (src/dd_bounds.h:442-479): can the side of `hand` (second to
// play) win this trick and, in NT, enough more? `t` is the trick-start table (the led card
// given back to the leader); `cutoff` counts this trick.
DDG_HD bool quick_tricks_2nd_impl(const u64* hands, const Top& t, int trump, int hand, int lead,
                             int cutoff, u64& wr) {
  int ls = card_suit(lead), P = partner_of(hand), L = lho_of(hand);
  u64 S = suit_cards(ls);
  u64 me = hand_at(hands, hand), pd = hand_at(hands, P), third = hand_at(hands, L);
  u64 ranks = (me | pd) & S;
  wr = 0;
  if (trump >= 0 && ls != trump) {
    u64 T = suit_cards(trump);
    bool we_ruff = (!(me & S) && (me & T)) || (!(pd & S) && (pd & T));
    bool they_ruff = !(third & S) && (third & T);
    if (we_ruff) {
      if (they_ruff) return false;
    } else if (ranks > (card_bit(lead) | (third & S))) {
      if (they_ruff) return false;
      wr = card_bit(top_bit(ranks));
    } else {
      return false;
    }
  } else if (ranks > (card_bit(lead) | (third & S))) {
    wr = card_bit(top_bit(ranks));
  } else {
    return false;
  }
  int qtricks = 1;
  if (qtricks >= cutoff) return true;
  if (trump >= 0) return false;
  int hh = (me & S) > (pd & S) ? hand : P;
  u64 mine = hand_at(hands, hh);
  if (winh(t, ls) == hh && sech(t, ls) == hh) {
    qtricks++;
    wr |= card_bit(secc(t, ls));
    if (qtricks >= cutoff) return true;
  }
  u64 others = all_cards(hands) & ~mine;
  for (int s = 0; s < 4; s++) {
    u64 m = mine & suit_cards(s);
    if (s == ls || !m) continue;
    if (!(others & suit_cards(s))) {
      qtricks += popc(m);
      if (qtricks >= cutoff) return true;
    } else if (winh(t, s) == hh) {
      qtricks++;
      wr |= card_bit(winc(t, s));
      if (qtricks >= cutoff) return true;
    }
  }
  return false;
}

// Longest holding of the partnership of seat hh in suit s.
DDG_HD int pair_len(const Top& t, int hh, int s) {
  int a = tlen(t, hh, s), b = tlen(t, partner_of(hh), s);
  return a > b ? a : b;
}
DDG_HD bool others_hold(const Top& t, int wh, int s) {
  return tlen(t, partner_of(wh), s) || tlen(t, lho_of(wh), s) || tlen(t, rho_of(wh), s);
}

// DDS LaterTricksMIN (src/dd_bounds.h:482-531), NS on lead: false = NS cannot reach
// `target` (wr = the cards that decided it).
DDG_HD bool later_min_impl(const Top& t, int trump, int hand, int ns_won, int left, int target,
                      u64& wr) {
  int dq = left - 1;
  if (trump < 0 || winh(t, trump) < 0) {
    int sum = 0;
    for (int s = 0; s < 4; s++) {
      int hh = winh(t, s);
      if (hh >= 0 && ns_side(hh)) sum += pair_len(t, hh, s);
    }
    if (ns_won + sum < target && sum > 0) {
      if (ns_won + dq >= target) return true;
      wr = 0;
      for (int s = 0; s < 4; s++) {
        int wh = winh(t, s);
        if (wh >= 0 && !ns_side(wh) && others_hold(t, wh, s)) wr |= card_bit(winc(t, s));
      }
      return false;
    }
    return true;
  }
  if (!ns_side(winh(t, trump))) {
    if (tlen(t, hand, trump) == 0 && tlen(t, partner_of(hand), trump) == 0) {
      int a = tlen(t, lho_of(hand), trump), b = tlen(t, rho_of(hand), trump);
      int m = a > b ? a : b;
      if (ns_won + dq + 1 - m < target) {
        wr = 0;
        return false;
      }
    } else if (ns_won + dq < target) {
      wr = card_bit(winc(t, trump));
      return false;
    } else if (ns_won + dq == target) {
      int hh = sech(t, trump);
      if (hh < 0) return true;
      if (!ns_side(hh) && (tlen(t, hh, trump) > 1 || tlen(t, partner_of(hh), trump) > 1)) {
        wr = card_bit(secc(t, trump));
        return false;
      }
    }
    return true;
  }
  int hh = sech(t, trump);
  if (hh < 0 || ns_side(hh) || tlen(t, hh, trump) <= 1) return true;
  if (winh(t, trump) == rho_of(hh)) {
    if (ns_won + dq < target) {
      wr = card_bit(secc(t, trump));
      return false;
    }
  } else {
    int h3 = thrh(t, trump);
    if (h3 < 0) return true;
    if (!ns_side(h3) && ns_won + dq < target) {
      wr = card_bit(thrc(t, trump));
      return false;
    }
  }
  return true;
}

// DDS LaterTricksMAX (src/dd_bounds.h:534-584), EW on lead: true = NS reach `target`.
DDG_HD bool later_max_impl(const Top& t, int trump, int hand, int ns_won, int left, int target,
                      u64& wr) {
  int dq = left - 1;
  if (trump < 0 || winh(t, trump) < 0) {
    int sum = 0;
    for (int s = 0; s < 4; s++) {
      int hh = winh(t, s);
      if (hh >= 0 && !ns_side(hh)) sum += pair_len(t, hh, s);
    }
    if (ns_won + dq + 1 - sum >= target && sum > 0) {
      if (ns_won + 1 < target) return false;
      wr = 0;
      for (int s = 0; s < 4; s++) {
        int wh = winh(t, s);
        if (wh >= 0 && ns_side(wh) && others_hold(t, wh, s)) wr |= card_bit(winc(t, s));
      }
      return true;
    }
    return false;
  }
  if (ns_side(winh(t, trump))) {
    if (tlen(t, hand, trump) == 0 && tlen(t, partner_of(hand), trump) == 0) {
      int a = tlen(t, lho_of(hand), trump), b = tlen(t, rho_of(hand), trump);
      int m = a > b ? a : b;
      if (ns_won + m >= target) {
        wr = 0;
        return true;
      }
    } else if (ns_won + 1 >= target) {
      wr = card_bit(winc(t, trump));
      return true;
    } else {
      int hh = sech(t, trump);
      if (hh < 0) return false;
      if (ns_side(hh) && (tlen(t, hh, trump) > 1 || tlen(t, partner_of(hh), trump) > 1) &&
          ns_won + 2 >= target) {
        wr = card_bit(secc(t, trump));
        return true;
      }
    }
    return false;
  }
  int hh = sech(t, trump);
  if (hh < 0 || !ns_side(hh) || tlen(t, hh, trump) <= 1) return false;
  if (winh(t, trump) == rho_of(hh)) {
    if (ns_won + 1 >= target) {
      wr = card_bit(secc(t, trump));
      return true;
    }
  } else {
    int h3 = thrh(t, trump);
    if (h3 < 0) return false;
    if (ns_side(h3) && ns_won + 1 >= target) {
      wr = card_bit(thrc(t, trump));
      return true;
    }
  }
  return false;
}

// Out-of-line entry points (arguments and results in registers).
DDG_CALL QtOut quick_tricks(Hands hs, Top t, int trump, int hand, int cutoff, int cutoff_other) {
  QtOut o;
  bool d = false;
  o.wr = 0;
  o.q = quick_tricks_impl(hs.h, t, trump, hand, cutoff, cutoff_other, o.wr, d);
  o.decided = d;
  return o;
}
DDG_CALL BoundOut quick_tricks_2nd(Hands hs, Top t, int trump, int hand, int lead, int cutoff) {
  BoundOut o;
  o.wr = 0;
  o.v = quick_tricks_2nd_impl(hs.h, t, trump, hand, lead, cutoff, o.wr);
  return o;
}
// LaterTricks for the side on lead: v = 1 when the bound decides the node (NS fail when
// NS lead, NS make it when EW lead).
DDG_CALL BoundOut later_tricks(Top t, int trump, int leader, int ns_won, int left, int target) {
  BoundOut o;
  o.wr = 0;
  o.v = ns_side(leader) ? !later_min_impl(t, trump, leader, ns_won, left, target, o.wr)
                        : later_max_impl(t, trump, leader, ns_won, left, target, o.wr);
  return o;
}

}  // namespace ddg
