"""shygpu: B200 implementation of SHYFEM's semi-implicit step (host side)."""
