cm = None
