// Move generation and DDS move ordering (src/dd.h:553-611, src/dd_bounds.h:586-949; the
// weights are DDS heuristic_sorting.cpp by Bo Haglund and Soren Hein, Apache-2.0). The
// scores, their constants and the tie order decide which child is searched first and so
// which nodes are visited; they are kept exactly. Tables live in packed registers.
#pragma once
#include "ddg_bounds.cuh"

namespace ddg {

// DDS rank scale: 2..14, 0 = no card.
DDG_HD int rank2(int card) { return (card & 15) + 2; }
DDG_HD int hi_rank(u64 m) { return m ? (top_bit(m) & 15) + 2 : 0; }
DDG_HD int lo_rank(u64 m) { return m ? (low_bit(m) & 15) + 2 : 0; }

// Two cards of one hand are alike when no card of another hand lies between them.
DDG_HD bool alike(u64 own, u64 all, int a, int b) {
  if (card_suit(a) != card_suit(b)) return false;
  int lo = a < b ? a : b, hi = a < b ? b : a;
  u64 between = (card_bit(hi) - 1) & ~(card_bit(lo + 1) - 1);
  return (all & ~own & between) == 0;
}

// Lead weight for `card` of hand `lead` (DDS weight_alloc_trump0 / weight_alloc_nt0).
// `tt` = the card, or one alike, is the TT's best move.
DDG_CALL int lead_weight(Hands hs, Top t, int trump, int left, int lead, int card, bool tt) {
  const u64* hands = hs.h;
  const int s = card_suit(card), P = partner_of(lead), L = lho_of(lead), R = rho_of(lead);
  const u64 S = suit_cards(s), all = all_cards(hands);
  const u64 hP = hand_at(hands, P), hL = hand_at(hands, L), hR = hand_at(hands, R);
  const int r_rank = popc(all & S & ~(card_bit(card) - 1));  // 1 = highest card of the suit
  const u64 below = all & S & (card_bit(card) - 1);
  const bool seq = below && ((hand_at(hands, lead) >> top_bit(below)) & 1);
  const u64 risP = hP & S, risL = hL & S, risR = hR & S;
  const int lenL = tlen(t, L, s), lenR = tlen(t, R, s), lenP = tlen(t, P, s);
  const int cnt = ((lenL == 0 ? left : lenL) << 2) + ((lenR == 0 ? left : lenR) << 2);
  const int w1 = winh(t, s), w2 = sech(t, s), w3 = thrh(t, s);
  int w;
  if (trump >= 0 && (all & suit_cards(trump))) {
    const u64 T = suit_cards(trump);
    const int tL = tlen(t, L, trump), tR = tlen(t, R, trump), tP = tlen(t, P, trump);
    const bool side = s != trump;
    int bonus = 0;
    if (side && ((!risL && (hL & T)) || (!risR && (hR & T)))) bonus = -12;
    if (side && lenP == 0 && tP > 0 && lenR > 0) bonus += 17;
    if (w1 == R || w2 == R) {
      if (lenR != 1) bonus -= 12;
    } else if (w1 == L && w2 == P) {
      if (lenP != 1) bonus += 27;
    }
    if (side && tlen(t, lead, s) == 1 && tlen(t, lead, trump) > 0 && lenP > 1 && w1 == P) bonus += 19;
    int delta = bonus - ((cnt << 5) / 13);
    bool win = false;
    if (winc(t, s) == card) {
      if (!side) {
        win = true;
      } else if (lenP != 0 || tP == 0) {
        win = (lenL != 0 || tL == 0) && (lenR != 0 || tR == 0);
      } else {
        win = (lenL != 0 || (hP & T) > (hL & T)) && (lenR != 0 || (hP & T) > (hR & T));
      }
    } else if (risP > (risL | risR)) {
      win = !side || ((lenL != 0 || tL == 0) && (lenR != 0 || tR == 0));
    } else if (side && lenP == 0 && tP != 0) {
      bool ruffL = lenL == 0 && tL != 0, ruffR = lenR == 0 && tR != 0;
      if (ruffL && ruffR) win = (hP & T) > ((hL | hR) & T);
      else if (ruffL) win = (hP & T) > (hL & T);
      else if (ruffR) win = (hP & T) > (hR & T);
      else win = true;
    }
    bool drop = (lenL == 1 && w1 == L) || (lenR == 1 && w1 == R);
    if (win) {
      if (drop) w = delta + 35 + r_rank;
      else if (w1 == lead) w = w2 == P ? delta + 48 + r_rank : winc(t, s) == card ? delta + 31 : delta - 3 + r_rank;
      else if (w1 == P) w = delta + (w2 == lead ? 42 : 28) + r_rank;
      else if (seq && card == secc(t, s)) w = delta + 40;
      else if (seq) w = delta + 22 + r_rank;
      else w = delta + 11 + r_rank;
      if (tt) w += 18;
    } else {
      if (w2 == P && P == w3) delta += 20;
      else if ((w2 == lead && P == w3 && lenP > 1) || (w2 == P && lead == w3 && lenP > 1)) delta += 13;
      if (drop) w = delta + r_rank + 2;
      else if (w1 == lead) w = w2 == P ? delta + 33 + r_rank : winc(t, s) == card ? delta + 38 : delta - 14 + r_rank;
      else if (w1 == P) w = delta + 34 + r_rank;
      else if (seq && card == secc(t, s)) w = delta + 35;
      else w = delta + 17 - rank2(card);
    }
    return w;
  }
  int delta = -((cnt << 5) / 19);
  if (lenP == 0) delta -= 9;
  if (winc(t, s) == card || risP > (risL | risR)) {
    if (w2 == R) {
      if (lenR != 1) delta -= 1;
    } else if (w2 == L) {
      delta += lenL != 1 ? 22 : 16;
    }
    w = ((w2 != L || lenL == 1) && (w2 != R || lenR == 1)) ? delta + 45 + r_rank : delta + 18 + r_rank;
    if (tt) w += 32;
  } else {
    if (w1 == R || w2 == R) {
      if (lenR != 1) delta -= 10;
    } else if (w1 == L && w2 == P) {
      if (lenP != 1) delta += 31;
    }
    if (w2 == P && P == w3) delta += 35;
    else if ((w2 == lead && P == w3 && lenP > 1) || (w2 == P && lead == w3 && lenP > 1)) delta += 25;
    if ((lenL == 1 && w1 == L) || (lenR == 1 && w1 == R)) w = delta + 28 + r_rank;
    else if (w1 == lead) w = delta - 17 + r_rank;
    else if (!seq) w = delta + 12 + r_rank;
    else if (card == secc(t, s)) w = delta + 48;
    else w = delta + 29 - r_rank;
    if (tt) w += 19;
  }
  return w;
}

DDG_HD bool beats(int card, int best, int trump) {
  int s = card_suit(card), bs = card_suit(best);
  return s == bs ? card > best : s == trump;
}
DDG_HD int trick_card(u32 trick, int i) { return (int)((trick >> (8 * i)) & 0xFF); }

// What the follow weights need about the trick so far, computed once per node.
struct Follow {
  u64 allt, all;       // all cards at the start of the trick / now
  u32 win_h, sec_h;    // byte s: trick-start holder of the top / second card of suit s
  int lead, ls, lead0;  // leader, led suit, led card's DDS rank
  int high1, move1, high2, move2;  // winner (index, card) after two and after three cards
};

DDG_HD Follow follow_init(const u64* hands, int trump, int leader, u32 trick, int n) {
  Follow f;
  u64 th[4] = {hands[0], hands[1], hands[2], hands[3]};
  for (int i = 0; i < n; i++) toggle_card(th, (leader + i) & 3, trick_card(trick, i));
  f.lead = leader;
  int c0 = trick_card(trick, 0);
  f.ls = card_suit(c0);
  f.all = all_cards(hands);
  f.allt = all_cards(th);
  f.win_h = f.sec_h = 0;
#pragma unroll
  for (int s = 0; s < 4; s++) {
    u64 m = f.allt & suit_cards(s);
    u32 a = 0xFF, b = 0xFF;
    if (m) {
      a = (u32)holder_of(th, top_bit(m));
      m &= ~card_bit(top_bit(m));
      if (m) b = (u32)holder_of(th, top_bit(m));
    }
    f.win_h |= a << (8 * s);
    f.sec_h |= b << (8 * s);
  }
  f.lead0 = rank2(c0);
  int c1 = trick_card(trick, 1), c2 = trick_card(trick, 2);
  int w1 = n > 1 && beats(c1, c0, trump) ? 1 : 0;
  int m1 = w1 ? c1 : c0;
  int w2 = n > 2 && beats(c2, m1, trump) ? 2 : w1;
  f.high1 = w1;
  f.move1 = m1;
  f.high2 = w2;
  f.move2 = w2 == 2 ? c2 : m1;
  return f;
}

// DDS weights for the 2nd, 3rd and 4th hand (weight_alloc_*1/2/3, without the
// rank_forces_ace / get_top_number bonuses); n = cards played to the trick so far.
DDG_CALL int follow_weight(Follow f, Hands hs, int trump, int n, int seat, int card) {
  const u64* hands = hs.h;
  const int lead = f.lead, ls = f.ls, lead0 = f.lead0;
  const u64 LS = suit_cards(ls);
  const int s = card_suit(card), rank = rank2(card);
  const int P = partner_of(lead), R = rho_of(lead);
  const u64 me = hand_at(hands, seat), hP = hand_at(hands, P), hR = hand_at(hands, R);
  const int r_rank = popc(f.all & suit_cards(s) & ~(card_bit(card) - 1));
  const u64 below = f.allt & suit_cards(s) & (card_bit(card) - 1);
  const bool seq = below && ((me >> top_bit(below)) & 1);
  const bool is_void = s != ls;
  const int sc = popc(me & suit_cards(s));
  const bool sec_mine = sbyte(f.sec_h, s) == seat, win_mine = sbyte(f.win_h, s) == seat;
  const u64 T = trump >= 0 ? suit_cards(trump) : 0;
  if (n == 1) {
    const int max3rd = hi_rank(hP & LS), maxpd = hi_rank(hR & LS);
    const int min3rd = lo_rank(hP & LS), minpd = lo_rank(hR & LS);
    if (!is_void) {
      if (trump >= 0) {
        bool win;
        if (ls == trump) {
          win = (maxpd > lead0 && maxpd > max3rd) || (rank > lead0 && rank > max3rd);
        } else if (rank > lead0 && rank > max3rd) {
          win = max3rd != 0 || !(hP & T) || (maxpd == 0 && (hR & T) && (hR & T) > (hP & T));
        } else if (maxpd > lead0 && maxpd > max3rd) {
          win = max3rd != 0 || !(hP & T);
        } else if (lead0 > maxpd && lead0 > max3rd && lead0 > rank) {
          win = maxpd == 0 && (hR & T) && (max3rd != 0 || !(hP & T) || (hR & T) > (hP & T));
        } else {
          win = maxpd == 0 && (hR & T);
        }
        if (win) {
          if (min3rd > rank) return 40 + r_rank;
          if (maxpd > lead0 && (hand_at(hands, lead) & LS) > (hR & LS)) return 41 + r_rank;
          if (rank > lead0) {
            if (rank < maxpd) return 78 - rank;
            if (rank > max3rd) return 73 - rank;
            return seq ? 62 - rank : 49 - rank;
          }
          return maxpd > 0 ? 47 - rank : 40 - rank;
        }
        if (rank < min3rd || rank < minpd) return -9 + r_rank;
        if (rank < lead0) return -16 + r_rank;
        return seq ? 22 - rank : 10 - rank;
      }
      if (maxpd > lead0 && maxpd > max3rd) return -rank;
      if (rank > lead0 && rank > max3rd) return 81 - rank;
      if (min3rd > rank || minpd > rank) return -3 + r_rank;
      if (rank < lead0) return -11 + r_rank;
      return seq ? 10 + r_rank : 13 - rank;
    }
    const u64 lead_bit = card_bit(ls * 16 + lead0 - 2);
    const bool r_over = (hR & LS) > ((hP & LS) | lead_bit);  // 4th hand beats the trick
    if (trump >= 0) {
      const int low_add = (sc << 6) / 36 - ((sc == 2 && sec_mine) ? 4 : 0);
      const int high_add = (sc << 6) / 44;
      if (ls == trump) return -rank + (r_over ? high_add : low_add);
      if (s != trump) {
        bool pd_wins;
        if (hP & LS) pd_wins = r_over || (!(hR & LS) && (hR & T));
        else pd_wins = (!(hR & LS) && (hR & T) > (hP & T)) || (!(hP & T) && (hR & LS) > lead_bit);
        return -rank + (pd_wins ? 60 + high_add : -2 + low_add);
      }
      if ((hP & LS) || (!(hR & LS) && (hR & T) && (hR & T) > (hP & T))) return 24 - rank + high_add;
      if (card_bit(card) > (hP & T)) return 24 - rank + high_add;
      return 15 - rank + low_add;
    }
    int add;
    if (r_over) {
      add = (sc << 6) / 23;
      if (sc == 2 && sec_mine) add -= 2;
      else if (sc == 1 && win_mine) add -= 3;
    } else {
      add = (sc << 6) / 33;
      if (sc == 2 && sec_mine) add -= 6;
      else if (sc == 1 && win_mine) add -= 8;
    }
    return -rank + add;
  }

  if (n == 2) {
    const u64 c4 = hR & LS;
    const int max4th = hi_rank(c4), min4th = lo_rank(c4);
    const int m1r = rank2(f.move1), m1s = card_suit(f.move1);
    if (!is_void) {
      const int max3rd = hi_rank(me & LS);
      if (trump >= 0 && ls != trump && m1s == trump) return -rank;
      if (trump >= 0 && ls != trump && f.high1 != 0 && max4th == 0) return rank > m1r ? 20 - rank : -rank;
      if (f.high1 == 0 && (lead0 > max4th || (trump >= 0 && ls != trump && max4th == 0))) return -rank;
      if (max3rd < min4th || max3rd < m1r) return -rank;
      if (trump >= 0 && max3rd > max4th) {
        if (ls == trump || f.high1 != 0) return rank > max4th && rank > m1r ? 58 - rank : -rank;
        return rank > max4th ? 58 - rank : -rank;
      }
      if (trump >= 0 && ls == trump) return -rank;
      return rank > m1r && rank > max4th ? 60 - rank : -rank;
    }
    if (trump >= 0) {
      if (ls == trump || s != trump) return -rank + (sc << 6) / 40;
      if (f.high1 == 0 && lead0 > max4th && (max4th != 0 || !(hR & T))) return -rank - 50;
      if (m1s == trump && rank < m1r) return -32 + r_rank + (sc << 6) / 40;
      const int add = (sc << 6) / 50;
      if (f.high1 == 0) {
        if (max4th != 0) return (sbyte(f.sec_h, ls) == lead ? 36 : 48) - rank + add;
        if (card_bit(card) > (hR & T)) return 48 - rank + add;
        return -12 - rank + add;
      }
      if (max4th != 0) return 72 - rank + add;
      if (card_bit(card) > (hR & T)) return 48 - rank + add;
      return 36 - rank + add;
    }
    int add = (sc << 6) / 24;
    if (sc == 2 && sec_mine) add -= 4;
    if (sc == 1 && win_mine) add -= 4;
    return -rank + add;
  }

  // Fourth hand.
  const int m2r = rank2(f.move2), m2s = card_suit(f.move2);
  if (!is_void) {
    if (f.high2 == 1 || (ls != trump && m2s == trump)) return -rank;
    return rank > m2r ? 30 - rank : -rank;
  }
  if (trump >= 0) {
    int val = (sc << 6) / 24;
    if (sc == 2 && sec_mine) val -= 2;
    if (ls == trump) return -rank + val;
    if (f.high2 == 1) return s == trump ? 2 - rank + val : 25 - rank + val;
    if (m2s == trump) {
      if (s == trump) return rank > m2r ? 33 + r_rank : -13 + r_rank;
      return 14 - rank + val;
    }
    if (s == trump) return 33 + r_rank;
    return 14 - rank + val;
  }
  int val = (sc << 6) / 27;
  if (sc == 2 && sec_mine) val -= 6;
  else if (sc == 1 && win_mine) val -= 8;
  return -rank + val;
}

// Cards of `own` that are the top of their run: a card is dropped when the next higher
// card still in play in its suit (`all` counts the cards of the current trick) is also
// in `own`. Computed for all suits at once by a log-step fill down through ranks no other
// hand holds; ranks 13..15 of each suit lane stop the fill.
DDG_HD u64 run_tops(u64 own, u64 all) {
  u64 open = ~(all & ~own) & 0x1FFF1FFF1FFF1FFFull;  // ranks a fill from above may cross
  u64 fill = own;
  fill |= open & (fill >> 1);
  open &= open >> 1;
  fill |= open & (fill >> 2);
  open &= open >> 2;
  fill |= open & (fill >> 4);
  open &= open >> 4;
  fill |= open & (fill >> 8);
  return own & ~(fill >> 1);
}

}  // namespace ddg
